"""GPU parity at the workloads the path is specified on, against the oracle.

* c1 splat forward + backward: 200,000 Gaussians with means in [-2, 2]^3,
  1024x1024, camera at distance 3 looking at the origin, upstream gradient
  N(0, 1) per pixel channel (seed 2);
* c2 vol_marcher forward + backward: 100,000 Gaussians, 512x512, float32;
* the served frame: 1,000,000 Gaussians (seed 0), 1920x1080, the first camera
  of random_cameras(seed=1) -- the frame the throughput number renders;
* a marcher frame whose tile lists exceed the 4096 entries the march keeps
  per-ray masks for, so the march re-tests entries past that point.

Bars (as in test_gpu_parity): bit-exact tile counts, offsets, rectangles,
keys, point lists, tile ranges and contributor counts; images within 1e-4
max-abs; gradients within 1e-3 per element, |gpu - cpu| / (|cpu| + 1e-3 max|cpu|).
The reference's code paths these follow: src/dgmr/splat_forward.cu:159-240,
src/dgmr/vol_marcher_forward.cu:340-490, src/dgmr/vol_marcher_backward.cu:172-317.
"""
import numpy as np
import pytest
import torch

from differentiable_gaussian_mixture_renderer_b200 import scene as S, splat
from oracle import oracle as O
from test_gpu_parity import GRAD_TOL, IMAGE_TOL, VM_NAMES, grad_err, run_splat, run_vm, to_dev, cam_tensors

pytestmark = pytest.mark.gpu

GRAD_NAMES = ("sh", "weights", "centroids", "scales", "rotations")


def check_splat_frame(fb, frame, ref):
    """Every binning output and the image of one splat frame against the oracle."""
    v = {k: t.cpu().numpy() for k, t in frame.views().items()}
    P = ref["n_pairs"]
    st = [int(x) for x in frame.stats.tolist()]
    assert st[0] == P and st[1] == 0, f"stats {st}, oracle pairs {P}"
    np.testing.assert_array_equal(v["tiles_touched"], ref["tiles_touched"])
    np.testing.assert_array_equal(v["point_offsets"], ref["point_offsets"])
    np.testing.assert_array_equal(v["rects"], ref["rects"])
    np.testing.assert_array_equal(v["i_ranges"], ref["i_ranges"])
    np.testing.assert_array_equal(v["point_list"][:P].astype(np.uint32), ref["point_list"])
    depth_bits = v["depths"].view(np.uint32)[v["point_list"][:P]]
    keys = (v["point_list_tiles"][:P].astype(np.uint64) << np.uint64(32)) | depth_bits.astype(np.uint64)
    np.testing.assert_array_equal(keys, ref["keys"])
    for k, ok in (("points_xy_image", "xy"), ("conic_opacity", "conic_opacity"), ("rgb", "rgb"), ("depths", "depths")):
        np.testing.assert_array_equal(v[k], ref[ok], err_msg=k)
    np.testing.assert_array_equal(v["rgb_sh_clamped"], ref["clamped"])
    np.testing.assert_array_equal(v["n_contrib"], ref["n_contrib"])
    assert np.abs(fb.cpu().numpy() - ref["fb"]).max() <= IMAGE_TOL
    assert np.abs(v["final_transmittance"] - ref["final_T"]).max() <= IMAGE_TOL
    return v


def test_c1_splat_forward_backward_200k_1024(cuda):
    sc = S.make_scene(200_000, seed=0, extent=2.0)
    cam = S.make_camera(1024, 1024)
    G = np.random.default_rng(2).normal(size=(3, cam.height, cam.width)).astype(np.float32)
    ref = O.splat_forward(sc, cam)
    gref = O.splat_backward(sc, cam, ref, G)
    fb, frame, ts = run_splat(sc, cam, cuda)
    check_splat_frame(fb, frame, ref)
    grads = splat.splat_backward(frame, torch.tensor(G, device=cuda), *ts)
    torch.cuda.synchronize()
    for name, g in zip(GRAD_NAMES, grads):
        e = grad_err(g.cpu().numpy().reshape(gref[name].shape), gref[name])
        assert e <= GRAD_TOL, (name, e)


def test_headline_frame_1080p_1M(cuda):
    """9.1M pairs over 8,160 tiles and 135 super-tiles whose lists run to many
    1024-entry chunks each."""
    sc = S.make_scene(1_000_000, seed=0)
    cam = S.random_cameras(1, 1920, 1080, seed=1)[0]
    ref = O.splat_forward(sc, cam)
    assert ref["n_pairs"] > 8_000_000
    fb, frame, _ = run_splat(sc, cam, cuda)
    check_splat_frame(fb, frame, ref)


def check_vm(sc, cam, dev, G, dtype=torch.float32):
    npdt = np.float32 if dtype == torch.float32 else np.float64
    with O.decision_audit() as audit:
        ref = O.vm_forward(sc, cam, dtype=npdt)
    cache, ts = run_vm(sc, cam, dev, dtype)
    # the march's work unit: (ray, Gaussian, large step) bin fills, counted by the kernel
    from differentiable_gaussian_mixture_renderer_b200 import cpp_binding
    counter = torch.zeros(1, dtype=torch.int64, device=dev)
    cpp_binding.forward(*ts[:5], *ts[5:9], cam.width, cam.height, cam.tan_fovx, cam.tan_fovy, sc.sh_degree,
                        work_counter=counter)
    assert int(counter.item()) == audit["fills"] > 0
    got = dict(zip(VM_NAMES, [c.cpu().numpy() for c in cache]))
    for k in ("rects", "tiles_touched", "point_offsets", "i_ranges", "b_point_list"):
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    np.testing.assert_array_equal(got["rgb_sh_clamped"].astype(np.uint8), ref["rgb_sh_clamped"])
    for k in ("rgb", "depths", "points_xy_image", "inverse_filtered_cov3d", "filtered_masses"):
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    assert np.abs(got["fb"] - ref["fb"]).max() <= IMAGE_TOL
    assert np.abs(got["remaining_transparency"] - ref["remaining_transparency"]).max() <= IMAGE_TOL
    gref = O.vm_backward(sc, cam, ref, G, dtype=npdt)
    shs, w, mu, s, q, view, proj, campos, bgt = ts
    grads = cpp_binding.backward(shs, w, mu, s, q, view, proj, campos, bgt, cam.width, cam.height, cam.tan_fovx,
                                 cam.tan_fovy, sc.sh_degree, torch.tensor(G, device=dev), cache)
    torch.cuda.synchronize()
    for name, g in zip(GRAD_NAMES, grads):
        e = grad_err(g.cpu().numpy().reshape(gref[name].shape), gref[name])
        assert e <= GRAD_TOL, (name, e)
    return ref


def test_c2_vol_marcher_forward_backward_100k_512(cuda):
    sc = S.make_scene(100_000, seed=0)
    cam = S.make_camera(512, 512)
    G = np.random.default_rng(2).normal(size=(3, 512, 512)).astype(np.float32)
    check_vm(sc, cam, cuda, G)


def test_vol_marcher_tile_lists_beyond_ray_masks(cuda):
    """A dense scene at a low resolution: some tile lists hold more than the
    4096 entries whose per-ray gate bits the march keeps in registers."""
    sc = S.make_scene(60_000, seed=4, sh_degree=1)
    cam = S.make_camera(96, 96)
    G = np.random.default_rng(5).normal(size=(3, 96, 96)).astype(np.float32)
    ref = check_vm(sc, cam, cuda, G)
    r = ref["i_ranges"].reshape(-1, 2)
    assert int((r[:, 1] - r[:, 0]).max()) > 4096


@pytest.mark.parametrize("steps", [4, 1])
def test_c2_step_store_gives_the_recomputed_results(cuda, steps):
    """The forward keeps the first `steps` large steps' samples of every ray and
    the backward reads them (steps beyond are recomputed): the image is the
    same bits and the gradients equal the recomputing backward's up to the
    order of the double-precision totals."""
    from differentiable_gaussian_mixture_renderer_b200 import cpp_binding
    sc = S.make_scene(100_000, seed=0)
    cam = S.random_cameras(1, 512, 512, seed=1)[0]
    G = torch.tensor(np.random.default_rng(2).normal(size=(3, 512, 512)).astype(np.float32), device=cuda)
    shs, w, mu, s, q = to_dev(sc, cuda)
    view, proj, campos, bgt = cam_tensors(cam, cuda)
    args = (shs, w, mu, s, q, view, proj, campos, bgt, 512, 512, cam.tan_fovx, cam.tan_fovy, 0)
    plain = cpp_binding.forward(*args)
    g_plain = cpp_binding.backward(*args, G, plain)
    store = cpp_binding.make_step_store(512, 512, steps, device=cuda)
    kept = cpp_binding.forward(*args, step_store=store)
    g_kept = cpp_binding.backward(*args, G, kept, step_store=store)
    torch.cuda.synchronize()
    assert torch.equal(plain[0], kept[0]) and torch.equal(plain[12], kept[12])
    for name, a, b in zip(GRAD_NAMES, g_kept, g_plain):
        err = float((a - b).abs().max()) / (float(b.abs().max()) + 1e-30)
        assert err <= 1e-5, (name, err)


def test_vol_marcher_apply_keeps_steps_when_memory_allows(cuda):
    """vol_marcher.apply stores the sample steps (memory is plentiful here) and
    gives the gradients of the recomputing path."""
    from differentiable_gaussian_mixture_renderer_b200 import vol_marcher
    sc = S.make_scene(20_000, seed=3, sh_degree=1)
    cam = S.make_camera(128, 96, eye=(0.3, -0.2, -3.0))
    G = torch.tensor(np.random.default_rng(4).normal(size=(3, 96, 128)).astype(np.float32), device=cuda)
    view, proj, campos, bgt = cam_tensors(cam, cuda)
    grads = []
    for steps in (vol_marcher.STORE_STEPS, 0):
        saved = vol_marcher.STORE_STEPS
        vol_marcher.STORE_STEPS = steps
        try:
            ins = [t.clone().requires_grad_(True) for t in to_dev(sc, cuda)]
            img = vol_marcher.apply(*ins, view, proj, campos, bgt, 128, 96, cam.tan_fovx, cam.tan_fovy, 1)
            (img * G).sum().backward()
            grads.append([t.grad for t in ins])
        finally:
            vol_marcher.STORE_STEPS = saved
    for name, a, b in zip(GRAD_NAMES, *grads):
        err = float((a - b).abs().max()) / (float(b.abs().max()) + 1e-30)
        assert err <= 1e-5, (name, err)
