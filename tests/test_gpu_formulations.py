"""The formulation switch (types.h:26-32; math.h:273-380, grad/math.h:284-527):
every renderer run with each formulation against the oracle run with the same
one.  Same bars as the default-formulation parity tests: bit-exact counts,
rectangles, order and per-Gaussian records, images within 1e-4, gradients
within 1e-3 of the oracle."""
import numpy as np
import pytest
import torch

from differentiable_gaussian_mixture_renderer_b200 import cpp_binding, scene as S, splat
from oracle import oracle as O

from test_gpu_parity import GRAD_TOL, IMAGE_TOL, VM_NAMES, cam_tensors, grad_err, to_dev

pytestmark = pytest.mark.gpu

FORMS = ["opacity", "mass", "density", "ots", "ols"]
NAMES = ("sh", "weights", "centroids", "scales", "rotations")


@pytest.mark.parametrize("form", FORMS)
def test_splat_forward_and_backward_per_formulation(cuda, form):
    sc = S.make_scene(3000, seed=11, extent=1.0, sh_degree=1)
    sc.formulation = form
    cam = S.make_camera(128, 96, eye=(0.3, -0.2, -3.0))
    bg = np.array((0.1, 0.2, 0.3), np.float32)
    ref = O.splat_forward(sc, cam, bg=bg)
    rng = np.random.default_rng(4)
    G = rng.normal(size=(3, cam.height, cam.width)).astype(np.float32)
    gref = O.splat_backward(sc, cam, ref, G, bg=bg)
    ts = to_dev(sc, cuda)
    view, proj, campos, bgt = cam_tensors(cam, cuda, bg=tuple(bg))
    fb, frame = splat.splat_forward(*ts, view, proj, campos, bgt, cam.width, cam.height, cam.tan_fovx, cam.tan_fovy,
                                    sc.sh_degree, formulation=form)
    torch.cuda.synchronize()
    v = {k: t.cpu().numpy() for k, t in frame.views().items()}
    P = ref["n_pairs"]
    assert int(frame.stats[0].item()) == P
    for k in ("tiles_touched", "point_offsets", "rects", "i_ranges"):
        np.testing.assert_array_equal(v[k], ref[k], err_msg=k)
    np.testing.assert_array_equal(v["point_list"][:P].astype(np.uint32), ref["point_list"])
    np.testing.assert_array_equal(v["conic_opacity"], ref["conic_opacity"])
    assert np.abs(fb.cpu().numpy() - ref["fb"]).max() <= IMAGE_TOL
    grads = splat.splat_backward(frame, torch.tensor(G, device=cuda), *ts)
    torch.cuda.synchronize()
    for name, g in zip(NAMES, grads):
        e = grad_err(g.cpu().numpy().reshape(gref[name].shape), gref[name])
        assert e <= GRAD_TOL, (form, name, e)


@pytest.mark.parametrize("form", FORMS)
def test_vol_marcher_forward_and_backward_per_formulation(cuda, form):
    sc = S.make_scene(1500, seed=12, sh_degree=1)
    sc.formulation = form
    cam = S.make_camera(48, 40, eye=(-0.2, 0.3, -3.0))
    bg = (0.3, 0.2, 0.1)
    rng = np.random.default_rng(6)
    G = rng.normal(size=(3, cam.height, cam.width)).astype(np.float32)
    ref = O.vm_forward(sc, cam, bg=np.array(bg, np.float32))
    gref = O.vm_backward(sc, cam, ref, G, bg=np.array(bg, np.float32))
    shs, w, mu, s, q = to_dev(sc, cuda)
    view, proj, campos, bgt = cam_tensors(cam, cuda, bg=bg)
    args = (shs, w, mu, s, q, view, proj, campos, bgt, cam.width, cam.height, cam.tan_fovx, cam.tan_fovy,
            sc.sh_degree)
    cache = cpp_binding.forward(*args, formulation=form)
    torch.cuda.synchronize()
    got = dict(zip(VM_NAMES, [c.cpu().numpy() for c in cache]))
    for k in ("rects", "tiles_touched", "point_offsets", "i_ranges", "b_point_list"):
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    np.testing.assert_array_equal(got["filtered_masses"], ref["filtered_masses"])
    assert np.abs(got["fb"] - ref["fb"]).max() <= IMAGE_TOL
    grads = cpp_binding.backward(*args, torch.tensor(G, device=cuda), cache, formulation=form)
    torch.cuda.synchronize()
    for name, g in zip(NAMES, grads):
        e = grad_err(g.cpu().numpy().reshape(gref[name].shape), gref[name])
        assert e <= GRAD_TOL, (form, name, e)


@pytest.mark.parametrize("form", FORMS)
def test_vol_raster_per_formulation(cuda, form):
    from differentiable_gaussian_mixture_renderer_b200 import vol_raster
    sc = S.make_scene(5000, seed=13, sh_degree=1)
    sc.formulation = form
    cam = S.make_camera(80, 64, eye=(0.2, 0.1, -3.0))
    bg = (0.1, 0.2, 0.3)
    ref = O.vr_forward(sc, cam, bg=np.array(bg, np.float32))
    shs, w, mu, s, q = to_dev(sc, cuda)
    view, proj, campos, bgt = cam_tensors(cam, cuda, bg=bg)
    fb = vol_raster.forward(shs, w, mu, s, q, view, proj, campos, bgt, cam.width, cam.height, cam.tan_fovx,
                            cam.tan_fovy, sc.sh_degree, formulation=form)
    assert np.abs(fb.cpu().numpy() - ref["fb"]).max() <= IMAGE_TOL


def test_batch_scene_formulations_equal_single_views(cuda):
    """Scenes of different formulations in one batched launch: every view
    equals the same view rendered alone with its scene's formulation."""
    from differentiable_gaussian_mixture_renderer_b200.batch import BatchRenderer
    from differentiable_gaussian_mixture_renderer_b200.serving import GaussianScene
    scenes = {}
    for k, form in enumerate(("mass", "opacity", None)):
        sc = S.make_scene(2000, seed=20 + k, sh_degree=1)
        sc.formulation = form
        scenes[str(form)] = GaussianScene.from_numpy(sc, cuda)
    views = [(sid, S.random_cameras(1, 64 + 16 * k, 48, seed=30 + k)[0]) for k, sid in enumerate(list(scenes) * 2)]
    r = BatchRenderer(scenes, cuda)
    p = r.plan(views)
    r.forward(p)
    torch.cuda.synchronize()
    for k, (sid, cam) in enumerate(views):
        g = scenes[sid]
        fb, _ = splat.splat_forward(g.shs, g.weights, g.centroids, g.scales, g.rotations, cam.view, cam.proj,
                                    cam.campos, (0.0, 0.0, 0.0), cam.width, cam.height, cam.tan_fovx, cam.tan_fovy,
                                    g.sh_degree, formulation=g.formulation)
        assert torch.equal(p.framebuffers[k], fb), (sid, k)
