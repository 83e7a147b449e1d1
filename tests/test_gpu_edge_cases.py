"""Edge cases on the GPU against the oracle: an empty scene (every renderer
draws the background; the marcher returns an empty point list and empty
gradients), and a scene with degenerate Gaussians mixed into ordinary ones --
zero scales (all three, or one axis), zero weights, unnormalised quaternions,
Gaussians at and behind the camera.  Same bars as the parity tests."""
import numpy as np
import pytest
import torch

from differentiable_gaussian_mixture_renderer_b200 import cpp_binding, scene as S, splat
from oracle import oracle as O

from test_gpu_parity import GRAD_TOL, IMAGE_TOL, VM_NAMES, cam_tensors, grad_err, to_dev

pytestmark = pytest.mark.gpu

BG = (0.1, 0.2, 0.3)
NAMES = ("sh", "weights", "centroids", "scales", "rotations")


def degenerate_scene():
    sc = S.make_scene(3000, seed=4, sh_degree=1)
    sc.scales[:50] = 0.0  # points
    sc.scales[50:100, 0] = 0.0  # flat along one axis
    sc.weights[100:150] = 0.0  # no opacity
    sc.rotations[150:200] *= 3.0  # quaternions of norm 3
    sc.centroids[200:220] = np.array([0.0, 0.0, -3.0])  # at the camera
    sc.centroids[220:240] = np.array([0.0, 0.0, -3.1])  # behind it
    return sc


def test_empty_scene_draws_the_background(cuda):
    sc = S.make_scene(0, seed=1)
    cam = S.make_camera(40, 32)
    shs, w, mu, s, q = to_dev(sc, cuda)
    view, proj, campos, bgt = cam_tensors(cam, cuda, bg=BG)
    fb, frame = splat.splat_forward(shs, w.reshape(-1), mu, s, q, view, proj, campos, bgt, cam.width, cam.height,
                                    cam.tan_fovx, cam.tan_fovy, 0)
    torch.cuda.synchronize()
    want = np.broadcast_to(np.array(BG, np.float32)[:, None, None], (3, cam.height, cam.width))
    np.testing.assert_array_equal(fb.cpu().numpy(), want)
    assert int(frame.stats[0].item()) == 0
    grads = splat.splat_backward(frame, torch.ones(3, cam.height, cam.width, device=cuda), shs, w.reshape(-1), mu, s, q)
    torch.cuda.synchronize()
    assert [tuple(g.shape) for g in grads] == [(0, 1, 3), (0,), (0, 3), (0, 3), (0, 4)]
    from differentiable_gaussian_mixture_renderer_b200 import vol_raster
    fr = vol_raster.forward(shs, w, mu, s, q, view, proj, campos, bgt, cam.width, cam.height, cam.tan_fovx, cam.tan_fovy, 0)
    np.testing.assert_array_equal(fr.cpu().numpy(), want)
    cache = cpp_binding.forward(shs, w, mu, s, q, view, proj, campos, bgt, cam.width, cam.height, cam.tan_fovx,
                                cam.tan_fovy, 0)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(cache[0].cpu().numpy(), want)
    np.testing.assert_array_equal(cache[12].cpu().numpy(), np.ones((cam.height, cam.width), np.float32))
    assert cache[11].numel() == 0
    grads = cpp_binding.backward(shs, w, mu, s, q, view, proj, campos, bgt, cam.width, cam.height, cam.tan_fovx,
                                 cam.tan_fovy, 0, torch.ones(3, cam.height, cam.width, device=cuda), cache)
    torch.cuda.synchronize()
    assert [tuple(g.shape) for g in grads] == [(0, 1, 3), (0, 1), (0, 3), (0, 3), (0, 4)]


def test_degenerate_gaussians_splat(cuda):
    sc = degenerate_scene()
    cam = S.make_camera(96, 80)
    bg = np.array(BG, np.float32)
    ref = O.splat_forward(sc, cam, bg=bg)
    G = np.random.default_rng(1).normal(size=(3, cam.height, cam.width)).astype(np.float32)
    gref = O.splat_backward(sc, cam, ref, G, bg=bg)
    ts = to_dev(sc, cuda)
    view, proj, campos, bgt = cam_tensors(cam, cuda, bg=BG)
    fb, frame = splat.splat_forward(*ts, view, proj, campos, bgt, cam.width, cam.height, cam.tan_fovx, cam.tan_fovy,
                                    sc.sh_degree)
    torch.cuda.synchronize()
    v = {k: t.cpu().numpy() for k, t in frame.views().items()}
    P = ref["n_pairs"]
    assert int(frame.stats[0].item()) == P
    for k in ("tiles_touched", "point_offsets", "rects", "i_ranges"):
        np.testing.assert_array_equal(v[k], ref[k], err_msg=k)
    np.testing.assert_array_equal(v["point_list"][:P].astype(np.uint32), ref["point_list"])
    out = fb.cpu().numpy()
    assert np.isfinite(out).all() and np.abs(out - ref["fb"]).max() <= IMAGE_TOL
    grads = splat.splat_backward(frame, torch.tensor(G, device=cuda), *ts)
    torch.cuda.synchronize()
    for name, g in zip(NAMES, grads):
        a = g.cpu().numpy().reshape(gref[name].shape)
        assert np.isfinite(a).all(), name
        assert grad_err(a, gref[name]) <= GRAD_TOL, name


def test_degenerate_gaussians_vol_marcher(cuda):
    sc = degenerate_scene()
    cam = S.make_camera(48, 40)
    bg = np.array(BG, np.float32)
    ref = O.vm_forward(sc, cam, bg=bg)
    G = np.random.default_rng(2).normal(size=(3, cam.height, cam.width)).astype(np.float32)
    gref = O.vm_backward(sc, cam, ref, G, bg=bg)
    shs, w, mu, s, q = to_dev(sc, cuda)
    view, proj, campos, bgt = cam_tensors(cam, cuda, bg=BG)
    args = (shs, w, mu, s, q, view, proj, campos, bgt, cam.width, cam.height, cam.tan_fovx, cam.tan_fovy, sc.sh_degree)
    cache = cpp_binding.forward(*args)
    torch.cuda.synchronize()
    got = dict(zip(VM_NAMES, [c.cpu().numpy() for c in cache]))
    for k in ("rects", "tiles_touched", "point_offsets", "i_ranges", "b_point_list"):
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    assert np.isfinite(got["fb"]).all() and np.abs(got["fb"] - ref["fb"]).max() <= IMAGE_TOL
    grads = cpp_binding.backward(*args, torch.tensor(G, device=cuda), cache)
    torch.cuda.synchronize()
    for name, g in zip(NAMES, grads):
        a = g.cpu().numpy().reshape(gref[name].shape)
        assert np.isfinite(a).all(), name
        assert grad_err(a, gref[name]) <= GRAD_TOL, name


def test_degenerate_gaussians_vol_raster(cuda):
    from differentiable_gaussian_mixture_renderer_b200 import vol_raster
    sc = degenerate_scene()
    cam = S.make_camera(64, 48)
    ref = O.vr_forward(sc, cam, bg=np.array(BG, np.float32))
    shs, w, mu, s, q = to_dev(sc, cuda)
    view, proj, campos, bgt = cam_tensors(cam, cuda, bg=BG)
    fb = vol_raster.forward(shs, w, mu, s, q, view, proj, campos, bgt, cam.width, cam.height, cam.tan_fovx,
                            cam.tan_fovy, sc.sh_degree).cpu().numpy()
    assert np.isfinite(fb).all() and np.abs(fb - ref["fb"]).max() <= IMAGE_TOL


def test_step_store_on_empty_and_degenerate_scenes(cuda):
    """The marcher's step store on an empty scene (every ray ends at its first
    step) and on the degenerate scene: the same image and gradients as the
    recomputing backward."""
    for sc in (S.make_scene(0, seed=1), degenerate_scene()):
        cam = S.make_camera(40, 32, eye=(0.1, -0.1, -3.0))
        ts = to_dev(sc, cuda)
        view, proj, campos, bgt = cam_tensors(cam, cuda, bg=BG)
        args = (*ts, view, proj, campos, bgt, cam.width, cam.height, cam.tan_fovx, cam.tan_fovy, sc.sh_degree)
        G = torch.tensor(np.random.default_rng(6).normal(size=(3, 32, 40)).astype(np.float32), device=cuda)
        plain = cpp_binding.forward(*args)
        g_plain = cpp_binding.backward(*args, G, plain)
        store = cpp_binding.make_step_store(cam.width, cam.height, 2, device=cuda)
        kept = cpp_binding.forward(*args, step_store=store)
        g_kept = cpp_binding.backward(*args, G, kept, step_store=store)
        torch.cuda.synchronize()
        assert torch.equal(plain[0], kept[0])
        for name, a, b in zip(NAMES, g_kept, g_plain):
            assert a.shape == b.shape
            if b.numel():
                err = float((a - b).abs().max()) / (float(b.abs().max()) + 1e-30)
                assert err <= 1e-5, (name, err)


def test_native_server_on_an_empty_and_a_culled_scene(cuda):
    """Scenes with no Gaussian, or none in front of the camera: splat and
    marcher requests, with gradients, complete with the background and the
    plain calls' (zero) gradients."""
    from differentiable_gaussian_mixture_renderer_b200.serving import GaussianScene, NativeServer, ServeRequest
    culled = S.make_scene(500, seed=11)
    culled.centroids[:, 2] -= 10.0
    scenes = {"empty": GaussianScene.from_numpy(S.make_scene(0, seed=1), cuda),
              "culled": GaussianScene.from_numpy(culled, cuda)}
    server = NativeServer(scenes, cuda, n_slots=2, max_batch=4)
    cam = S.make_camera(48, 40)
    reqs = []
    for sid in ("empty", "culled"):
        for kind in ("splat", "march"):
            g = torch.ones((3, 40, 48), device=cuda)
            reqs.append(server.submit(ServeRequest(sid, cam, backward=True, grad_image=g, kind=kind)))
    server.drain()
    want = torch.zeros((3, 40, 48), device=cuda)  # camera_struct's background is black
    for r in reqs:
        assert r.status == 0
        assert torch.equal(r.image, want)
        for g in r.grads:
            assert g.numel() == 0 or float(g.abs().max()) == 0.0
    server.close()
