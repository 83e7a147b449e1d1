"""GPU kernels (through the C ABI) against the CPU oracle on seeded scenes.

Bars: bit-exact tile counts, offsets, rectangles, sort keys, sorted order and
tile ranges; images within 1e-4 max-abs (float32); gradients within 1e-3 of
the oracle, measured per element as |gpu - cpu| / (|cpu| + 1e-3 * max|cpu|).
"""
import numpy as np
import pytest
import torch

from differentiable_gaussian_mixture_renderer_b200 import cpp_binding, scene as S, splat
from oracle import oracle as O

pytestmark = pytest.mark.gpu

IMAGE_TOL = 1e-4
GRAD_TOL = 1e-3


def to_dev(sc, dev, dtype=torch.float32):
    t = lambda a: torch.tensor(np.ascontiguousarray(a), dtype=dtype, device=dev)
    return t(sc.sh), t(sc.weights).reshape(-1, 1), t(sc.centroids), t(sc.scales), t(sc.rotations)


def cam_tensors(cam, dev, dtype=torch.float32, bg=(0.0, 0.0, 0.0)):
    t = lambda a: torch.tensor(np.asarray(a), dtype=dtype, device=dev)
    return t(cam.view), t(cam.proj), t(cam.campos), t(bg)


def grad_err(gpu, cpu):
    gpu = np.asarray(gpu, dtype=np.float64)
    cpu = np.asarray(cpu, dtype=np.float64)
    scale = np.abs(cpu).max() if cpu.size else 0.0
    if scale == 0.0:
        return float(np.abs(gpu).max()) if gpu.size else 0.0
    return float((np.abs(gpu - cpu) / (np.abs(cpu) + 1e-3 * scale)).max())


def run_splat(sc, cam, dev, bg=(0.0, 0.0, 0.0)):
    shs, w, mu, s, q = to_dev(sc, dev)
    view, proj, campos, bgt = cam_tensors(cam, dev, bg=bg)
    fb, frame = splat.splat_forward(shs, w, mu, s, q, view, proj, campos, bgt, cam.width, cam.height, cam.tan_fovx,
                                    cam.tan_fovy, sc.sh_degree)
    torch.cuda.synchronize()
    return fb, frame, (shs, w, mu, s, q)


@pytest.mark.parametrize("n,w,h,seed,extent", [(10000, 256, 256, 0, 1.0), (3000, 200, 120, 7, 1.5), (1, 40, 33, 3, 0.2)])
def test_splat_forward_bit_exact(cuda, n, w, h, seed, extent):
    sc = S.make_scene(n, seed=seed, extent=extent)
    cam = S.make_camera(w, h)
    ref = O.splat_forward(sc, cam)
    fb, frame, _ = run_splat(sc, cam, cuda)
    v = {k: t.cpu().numpy() for k, t in frame.views().items()}
    P = ref["n_pairs"]
    st = [int(v) for v in frame.stats.tolist()]
    assert st[0] == P and st[1] == 0, f"stats {st}, oracle pairs {P}"
    np.testing.assert_array_equal(v["tiles_touched"], ref["tiles_touched"])
    np.testing.assert_array_equal(v["point_offsets"], ref["point_offsets"])
    np.testing.assert_array_equal(v["rects"], ref["rects"])
    np.testing.assert_array_equal(v["i_ranges"], ref["i_ranges"])
    np.testing.assert_array_equal(v["point_list"][:P].astype(np.uint32), ref["point_list"])
    # the sort keys: tile id in the high word, float bits of the depth in the low word
    depth_bits = v["depths"].view(np.uint32)[v["point_list"][:P]]
    keys = (v["point_list_tiles"][:P].astype(np.uint64) << np.uint64(32)) | depth_bits.astype(np.uint64)
    np.testing.assert_array_equal(keys, ref["keys"])
    for k in ("points_xy_image", "conic_opacity", "rgb", "depths"):
        ok = {"points_xy_image": "xy", "conic_opacity": "conic_opacity", "rgb": "rgb", "depths": "depths"}[k]
        np.testing.assert_array_equal(v[k], ref[ok], err_msg=k)
    np.testing.assert_array_equal(v["rgb_sh_clamped"], ref["clamped"])
    img = fb.cpu().numpy()
    assert np.abs(img - ref["fb"]).max() <= IMAGE_TOL
    np.testing.assert_array_equal(v["n_contrib"], ref["n_contrib"])
    assert np.abs(v["final_transmittance"] - ref["final_T"]).max() <= IMAGE_TOL


def test_splat_forward_background_and_culled(cuda):
    sc = S.make_scene(500, seed=11)
    sc.centroids[:, 2] -= 10.0  # everything behind the camera: no pairs at all
    cam = S.make_camera(64, 48)
    fb, frame, _ = run_splat(sc, cam, cuda, bg=(0.25, 0.5, 0.75))
    assert int(frame.stats[0]) == 0
    img = fb.cpu().numpy()
    np.testing.assert_allclose(img[0], 0.25)
    np.testing.assert_allclose(img[2], 0.75)


def test_splat_pair_overflow_is_flagged(cuda):
    sc = S.make_scene(2000, seed=1)
    cam = S.make_camera(128, 128)
    shs, w, mu, s, q = to_dev(sc, cuda)
    view, proj, campos, bg = cam_tensors(cam, cuda)
    ref = O.splat_forward(sc, cam, want_keys=False)
    fb, frame = splat.splat_forward(shs, w, mu, s, q, view, proj, campos, bg, cam.width, cam.height, cam.tan_fovx,
                                    cam.tan_fovy, 0, pair_capacity=100)
    torch.cuda.synchronize()
    assert int(frame.stats[0]) == ref["n_pairs"] and int(frame.stats[1]) & 1
    # the retrying call sizes itself and matches
    fb2, frame2, _ = run_splat(sc, cam, cuda)
    assert np.abs(fb2.cpu().numpy() - ref["fb"]).max() <= IMAGE_TOL


# 150 x 93: the frame's last tile row and column hold partial 8x8 blend blocks
# and whole blocks outside the frame
@pytest.mark.parametrize("w,h", [(160, 128), (150, 93)])
def test_splat_backward_matches_oracle(cuda, w, h):
    sc = S.make_scene(4000, seed=5, extent=1.0, sh_degree=2)
    cam = S.make_camera(w, h, eye=(0.4, -0.3, -3.0))
    rng = np.random.default_rng(2)
    G = rng.normal(size=(3, cam.height, cam.width)).astype(np.float32)
    bg = (0.1, 0.2, 0.3)
    ref = O.splat_forward(sc, cam, bg=np.array(bg, np.float32))
    gref = O.splat_backward(sc, cam, ref, G, bg=np.array(bg, np.float32))
    fb, frame, ts = run_splat(sc, cam, cuda, bg=bg)
    assert np.abs(fb.cpu().numpy() - ref["fb"]).max() <= IMAGE_TOL
    grads = splat.splat_backward(frame, torch.tensor(G, device=cuda), *ts)
    torch.cuda.synchronize()
    names = ("sh", "weights", "centroids", "scales", "rotations")
    for name, g in zip(names, grads):
        e = grad_err(g.cpu().numpy().reshape(gref[name].shape), gref[name])
        assert e <= GRAD_TOL, (name, e)


def run_vm(sc, cam, dev, dtype, bg=(0.0, 0.0, 0.0)):
    shs, w, mu, s, q = to_dev(sc, dev, dtype)
    view, proj, campos, bgt = cam_tensors(cam, dev, dtype, bg)
    cache = cpp_binding.forward(shs, w, mu, s, q, view, proj, campos, bgt, cam.width, cam.height, cam.tan_fovx,
                                cam.tan_fovy, sc.sh_degree)
    torch.cuda.synchronize()
    return cache, (shs, w, mu, s, q, view, proj, campos, bgt)


VM_NAMES = ("fb", "rects", "rgb", "rgb_sh_clamped", "depths", "points_xy_image", "inverse_filtered_cov3d",
            "filtered_masses", "tiles_touched", "point_offsets", "i_ranges", "b_point_list", "remaining_transparency")


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
@pytest.mark.parametrize("n,w,h,seed", [(3000, 64, 64, 0), (800, 50, 37, 4)])
def test_vol_marcher_forward_matches_oracle(cuda, dtype, n, w, h, seed):
    npdt = np.float32 if dtype == torch.float32 else np.float64
    sc = S.make_scene(n, seed=seed, sh_degree=1)
    cam = S.make_camera(w, h, eye=(0.3, 0.2, -3.0))
    bg = (0.2, 0.1, 0.4)
    ref = O.vm_forward(sc, cam, bg=np.array(bg, npdt), dtype=npdt)
    cache, _ = run_vm(sc, cam, cuda, dtype, bg)
    got = dict(zip(VM_NAMES, [c.cpu().numpy() for c in cache]))
    for k in ("rects", "tiles_touched", "point_offsets", "i_ranges", "b_point_list"):
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    np.testing.assert_array_equal(got["rgb_sh_clamped"].astype(np.uint8), ref["rgb_sh_clamped"])
    for k in ("rgb", "depths", "points_xy_image", "inverse_filtered_cov3d", "filtered_masses"):
        np.testing.assert_array_equal(got[k], ref[k], err_msg=k)
    assert np.abs(got["fb"] - ref["fb"]).max() <= IMAGE_TOL
    assert np.abs(got["remaining_transparency"] - ref["remaining_transparency"]).max() <= IMAGE_TOL


@pytest.mark.parametrize("mode,code", [("bins", 1), ("depth", 2)])
def test_vol_marcher_debug_modes_match_oracle(cuda, mode, code):
    """vol_marcher_forward.cu:448-482: Bins (one bin's channel sum of the first
    large step) and Depth (distance marched, inf while the section set is open)."""
    sc = S.make_scene(20000, seed=6, sh_degree=0)
    cam = S.make_camera(40, 32, eye=(0.1, -0.2, -3.0))
    ref = O.vm_forward(sc, cam, render_mode=code, debug_bin=30, max_depth=10.0)
    O.vm_forward(sc, cam)  # back to Full for the other tests
    shs, w, mu, s, q = to_dev(sc, cuda, torch.float32)
    view, proj, campos, bgt = cam_tensors(cam, cuda, torch.float32, (0.0, 0.0, 0.0))
    cache = cpp_binding.forward(shs, w, mu, s, q, view, proj, campos, bgt, cam.width, cam.height, cam.tan_fovx,
                                cam.tan_fovy, sc.sh_degree, render_mode=mode, debug_render_bin=30, max_depth=10.0)
    got = cache[0].cpu().numpy()
    np.testing.assert_array_equal(np.isinf(got), np.isinf(ref["fb"]))
    fin = np.isfinite(ref["fb"])
    if fin.any():
        assert np.abs(got[fin] - ref["fb"][fin]).max() <= IMAGE_TOL
    np.testing.assert_array_equal(cache[12].cpu().numpy(), ref["remaining_transparency"])


@pytest.mark.parametrize("dtype", [torch.float32, torch.float64])
def test_vol_marcher_backward_matches_oracle(cuda, dtype):
    npdt = np.float32 if dtype == torch.float32 else np.float64
    sc = S.make_scene(1500, seed=3, sh_degree=2)
    cam = S.make_camera(48, 40, eye=(-0.2, 0.3, -3.0))
    bg = (0.3, 0.2, 0.1)
    rng = np.random.default_rng(2)
    G = rng.normal(size=(3, cam.height, cam.width)).astype(npdt)
    ref = O.vm_forward(sc, cam, bg=np.array(bg, npdt), dtype=npdt)
    gref = O.vm_backward(sc, cam, ref, G, bg=np.array(bg, npdt), dtype=npdt)
    cache, ts = run_vm(sc, cam, cuda, dtype, bg)
    shs, w, mu, s, q, view, proj, campos, bgt = ts
    grads = cpp_binding.backward(shs, w, mu, s, q, view, proj, campos, bgt, cam.width, cam.height, cam.tan_fovx,
                                 cam.tan_fovy, sc.sh_degree, torch.tensor(G, device=cuda), cache)
    torch.cuda.synchronize()
    for name, g in zip(("sh", "weights", "centroids", "scales", "rotations"), grads):
        e = grad_err(g.cpu().numpy().reshape(gref[name].shape), gref[name])
        assert e <= GRAD_TOL, (name, e)


def test_splat_large_frame_bit_exact(cuda):
    """A 4096x2304 frame: 36,864 tiles (the three-launch tile scan, above the
    one-block limit) and 576 super-tiles (two radix passes over the super-tile
    entries instead of one) -- the point list, its tile ids, the ranges and
    the image against the oracle."""
    sc = S.make_scene(200_000, seed=9, extent=1.0)
    cam = S.make_camera(4096, 2304, eye=(0.2, -0.1, -2.6))
    ref = O.splat_forward(sc, cam)
    fb, frame, _ = run_splat(sc, cam, cuda)
    v = {k: t.cpu().numpy() for k, t in frame.views().items()}
    P = ref["n_pairs"]
    st = [int(x) for x in frame.stats.tolist()]
    assert st[0] == P and st[1] == 0, f"stats {st}, oracle pairs {P}"
    np.testing.assert_array_equal(v["i_ranges"], ref["i_ranges"])
    np.testing.assert_array_equal(v["point_list"][:P].astype(np.uint32), ref["point_list"])
    depth_bits = v["depths"].view(np.uint32)[v["point_list"][:P]]
    keys = (v["point_list_tiles"][:P].astype(np.uint64) << np.uint64(32)) | depth_bits.astype(np.uint64)
    np.testing.assert_array_equal(keys, ref["keys"])
    assert np.abs(fb.cpu().numpy() - ref["fb"]).max() <= IMAGE_TOL
