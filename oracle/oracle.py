"""TEST INFRASTRUCTURE ONLY: ctypes wrapper of the CPU oracle library.

Only tests/, bench.py's CPU-baseline legs and __graft_entry__.smoke() import
this module; the product package never does.  Every function takes numpy
arrays in the reference's layouts and returns numpy arrays.
"""
from __future__ import annotations

import contextlib
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libdgmr_oracle.so")
# the same restatement with the host libm's expf / logf / erff (see libm_transcendentals)
_LIBM_PATH = os.path.join(_HERE, "_build", "libdgmr_oracle_libm.so")
_libs: dict = {}
_variant = _LIB_PATH

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_u64p = np.ctypeslib.ndpointer(np.uint64, flags="C_CONTIGUOUS")
_u8p = np.ctypeslib.ndpointer(np.uint8, flags="C_CONTIGUOUS")


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    if _variant not in _libs:
        if not os.path.exists(_variant):
            build()
        L = C.CDLL(_variant)
        _declare(L)
        _libs[_variant] = L
    return _libs[_variant]


@contextlib.contextmanager
def libm_transcendentals():
    """Inside this block every oracle call runs the build whose exp / log /
    erf are the host C library's (correctly rounded or nearly so) instead of
    the fixed-sequence routines the CUDA kernels share with the default
    build: the closest stand-in available here for the CUDA expf / erff the
    reference calls.  Used to measure what sharing those routines hides."""
    global _variant
    old = _variant
    _variant = _LIBM_PATH
    try:
        yield
    finally:
        _variant = old


def _scene_types(fp):
    return [C.c_int, fp, fp, C.c_int, C.c_int, fp, fp, fp, fp, fp, fp, fp, C.c_int, C.c_int,
            C.c_float if fp is _f32p else C.c_double, C.c_float if fp is _f32p else C.c_double,
            C.c_float if fp is _f32p else C.c_double]


def _declare(L):
    L.orc_audit.argtypes = [C.c_int, C.POINTER(C.c_long)]
    L.orc_audit.restype = None
    L.orc_num_threads.restype = C.c_int
    L.orc_set_num_threads.argtypes = [C.c_int]
    L.orc_higher_msb.restype = C.c_uint32
    L.orc_higher_msb.argtypes = [C.c_uint32]
    L.orc_splat_forward_f32.restype = C.c_int64
    L.orc_splat_forward_f32.argtypes = _scene_types(_f32p) + [
        _f32p, _i32p, _f32p, _u8p, _f32p, _f32p, _f32p, _i32p, _i32p, _i32p,
        C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
    L.orc_vr_forward_f32.restype = C.c_int64
    L.orc_vr_forward_f32.argtypes = _scene_types(_f32p) + [
        _f32p, _i32p, _f32p, _u8p, _f32p, _f32p, _f32p, _f32p, _i32p, _i32p, _i32p, C.c_void_p, C.c_int64]
    L.orc_splat_backward_f32.restype = None
    L.orc_splat_backward_f32.argtypes = _scene_types(_f32p) + [
        _f32p, _u8p, _f32p, _f32p, _i32p, _i32p, _u32p, _f32p, _i32p, _f32p,
        _f32p, _f32p, _f32p, _f32p, _f32p]
    L.orc_splat_render_f64.restype = None
    L.orc_splat_render_f64.argtypes = _scene_types(_f64p) + [
        _f64p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    for sfx, fp in (("f32", _f32p), ("f64", _f64p)):
        cache = [fp, _i32p, fp, _u8p, fp, fp, fp, fp, _i32p, _i32p, _i32p, fp]
        f = getattr(L, f"orc_vm_preprocess_{sfx}")
        f.restype = C.c_int64
        f.argtypes = _scene_types(fp) + cache
        f = getattr(L, f"orc_vm_render_{sfx}")
        f.restype = C.c_int32
        f.argtypes = _scene_types(fp) + cache + [_i32p, C.c_void_p]
        f = getattr(L, f"orc_vm_backward_{sfx}")
        f.restype = C.c_int32
        f.argtypes = _scene_types(fp) + cache + [_i32p, fp, fp, fp, fp, fp, fp]
        f = getattr(L, f"orc_density_array_{sfx}")
        f.restype = C.c_int
        f.argtypes = [C.c_int, C.c_float if sfx == "f32" else C.c_double, fp, C.c_int, fp, fp]
        f = getattr(L, f"orc_density_combine_{sfx}")
        f.restype = None
        f.argtypes = [fp, fp, fp]
        f = getattr(L, f"orc_density_sample_{sfx}")
        f.restype = None
        f.argtypes = [C.c_int, C.c_float if sfx == "f32" else C.c_double, fp, C.c_int, C.c_int, fp]
    for sfx in ("f32", "f64"):
        f = getattr(L, f"orc_density_randomised_{sfx}")
        f.restype = C.c_int
        f.argtypes = [C.c_int, C.c_int, C.c_int]
    L.orc_set_formulation.restype = None
    L.orc_set_formulation.argtypes = [C.c_int]
    L.orc_set_render_mode.restype = None
    L.orc_set_render_mode.argtypes = [C.c_int, C.c_int, C.c_double]
    L.orc_set_const_samples.restype = None
    L.orc_set_const_samples.argtypes = [C.c_int, _f64p]
    L.orc_fmath_f32.restype = None
    L.orc_fmath_f32.argtypes = [C.c_int, _f32p, _f32p, C.c_int]
    L.orc_pick2_f32.restype = None
    L.orc_pick2_f32.argtypes = [C.c_int, _f32p, _f32p, C.c_int]


def num_threads() -> int:
    return lib().orc_num_threads()


def set_num_threads(n: int) -> None:
    lib().orc_set_num_threads(int(n))


def higher_msb(n: int) -> int:
    return int(lib().orc_higher_msb(n))


def _c(a, dt):
    return np.ascontiguousarray(a, dtype=dt)


_FORMS = {None: 0, "opacity": 1, "mass": 2, "density": 3, "ots": 4, "ols": 5}


def _scene_args(scene, cam, dt, bg=None, cov_mult=1.0):
    """The scene/camera arguments of every oracle entry point; also selects the
    scene's formulation (attribute 'formulation': None = the renderer's
    reference default, or opacity/mass/density/ots/ols) for the call."""
    lib().orc_set_formulation(_FORMS[getattr(scene, "formulation", None)])
    sh = _c(scene.sh, dt)
    bg = np.zeros(3, dt) if bg is None else _c(bg, dt)
    return [scene.n, _c(scene.centroids, dt), sh, sh.shape[1], scene.sh_degree, _c(scene.weights, dt).reshape(-1),
            _c(scene.scales, dt), _c(scene.rotations, dt), _c(cam.view, dt), _c(cam.proj, dt), _c(cam.campos, dt), bg,
            cam.width, cam.height, cam.tan_fovx, cam.tan_fovy, cov_mult]


def tiles(cam):
    return (cam.width + 15) // 16, (cam.height + 15) // 16


def splat_forward(scene, cam, bg=None, cov_mult=1.0, want_keys=True):
    """Reference-order splat forward.  Returns a dict of numpy outputs."""
    L = lib()
    N, W, H = scene.n, cam.width, cam.height
    gx, gy = tiles(cam)
    out = dict(fb=np.zeros((3, H, W), np.float32), rects=np.zeros((N, 2), np.int32), rgb=np.zeros((N, 3), np.float32),
               clamped=np.zeros((N, 3), np.uint8), depths=np.zeros(N, np.float32), xy=np.zeros((N, 2), np.float32),
               conic_opacity=np.zeros((N, 4), np.float32), tiles_touched=np.zeros(N, np.int32),
               point_offsets=np.zeros(N, np.int32), i_ranges=np.zeros((gx * gy, 2), np.int32),
               final_T=np.zeros((H, W), np.float32), n_contrib=np.zeros((H, W), np.int32))
    args = _scene_args(scene, cam, np.float32, bg, cov_mult)
    outs = [out[k] for k in ("fb", "rects", "rgb", "clamped", "depths", "xy", "conic_opacity", "tiles_touched",
                             "point_offsets", "i_ranges")]
    P = int(out["point_offsets"][-1]) if N else 0
    keys = np.zeros(max(1, 1), np.uint64)
    vals = np.zeros(1, np.uint32)
    cap = 0
    if want_keys:
        # first pass sizes the pair buffers
        P = L.orc_splat_forward_f32(*args, *outs, None, None, 0, None, None)
        keys = np.zeros(max(P, 1), np.uint64)
        vals = np.zeros(max(P, 1), np.uint32)
        cap = P
    P = L.orc_splat_forward_f32(*args, *outs, keys.ctypes.data, vals.ctypes.data, cap,
                                out["final_T"].ctypes.data, out["n_contrib"].ctypes.data)
    out["n_pairs"] = P
    if want_keys:
        out["keys"] = keys[:P]
        out["point_list"] = vals[:P]
    return out


def splat_backward(scene, cam, fwd, grad_fb, bg=None, cov_mult=1.0):
    L = lib()
    N = scene.n
    k = scene.sh.shape[1]
    g = dict(sh=np.zeros((N, k, 3), np.float32), weights=np.zeros(N, np.float32), centroids=np.zeros((N, 3), np.float32),
             scales=np.zeros((N, 3), np.float32), rotations=np.zeros((N, 4), np.float32))
    L.orc_splat_backward_f32(*_scene_args(scene, cam, np.float32, bg, cov_mult), fwd["rgb"], fwd["clamped"], fwd["xy"],
                             fwd["conic_opacity"], fwd["tiles_touched"], fwd["i_ranges"], _c(fwd["point_list"], np.uint32),
                             fwd["final_T"], fwd["n_contrib"], _c(grad_fb, np.float32), g["sh"], g["weights"],
                             g["centroids"], g["scales"], g["rotations"])
    return g


def splat_render_f64(scene, cam, grad_fb=None, bg=None, cov_mult=1.0):
    """Double-precision splat forward (and backward when grad_fb is given)."""
    L = lib()
    N, W, H = scene.n, cam.width, cam.height
    fb = np.zeros((3, H, W), np.float64)
    k = scene.sh.shape[1]
    g = dict(sh=np.zeros((N, k, 3)), weights=np.zeros(N), centroids=np.zeros((N, 3)), scales=np.zeros((N, 3)),
             rotations=np.zeros((N, 4)))
    gp = None if grad_fb is None else _c(grad_fb, np.float64)
    ptr = lambda a: a.ctypes.data
    L.orc_splat_render_f64(*_scene_args(scene, cam, np.float64, bg, cov_mult), fb,
                           None if gp is None else ptr(gp), ptr(g["sh"]), ptr(g["weights"]), ptr(g["centroids"]),
                           ptr(g["scales"]), ptr(g["rotations"]))
    return (fb, g) if grad_fb is not None else fb


def _vm_cache(N, W, H, gx, gy, dt):
    return dict(fb=np.zeros((3, H, W), dt), rects=np.zeros((N, 2), np.int32), rgb=np.zeros((N, 3), dt),
                rgb_sh_clamped=np.zeros((N, 3), np.uint8), depths=np.zeros(N, dt), points_xy_image=np.zeros((N, 2), dt),
                inverse_filtered_cov3d=np.zeros((N, 6), dt), filtered_masses=np.zeros(N, dt),
                tiles_touched=np.zeros(N, np.int32), point_offsets=np.zeros(N, np.int32),
                i_ranges=np.zeros((gx * gy, 2), np.int32), remaining_transparency=np.zeros((H, W), dt))


_VM_ORDER = ("fb", "rects", "rgb", "rgb_sh_clamped", "depths", "points_xy_image", "inverse_filtered_cov3d",
             "filtered_masses", "tiles_touched", "point_offsets", "i_ranges", "remaining_transparency")


def vr_forward(scene, cam, bg=None, cov_mult=1.0, want_list=False):
    """vol_raster forward (float32).  Returns a dict of numpy outputs: the
    framebuffer and the per-Gaussian preprocess, ranges and (optionally) the
    sorted point list."""
    L = lib()
    N, W, H = scene.n, cam.width, cam.height
    gx, gy = tiles(cam)
    out = dict(fb=np.zeros((3, H, W), np.float32), rects=np.zeros((N, 2), np.int32), rgb=np.zeros((N, 3), np.float32),
               clamped=np.zeros((N, 3), np.uint8), depths=np.zeros(N, np.float32), xy=np.zeros((N, 2), np.float32),
               inverse_filtered_cov3d=np.zeros((N, 6), np.float32), filtered_masses=np.zeros(N, np.float32),
               tiles_touched=np.zeros(N, np.int32), point_offsets=np.zeros(N, np.int32),
               i_ranges=np.zeros((gx * gy, 2), np.int32))
    args = _scene_args(scene, cam, np.float32, bg, cov_mult)
    outs = [out[k] for k in ("fb", "rects", "rgb", "clamped", "depths", "xy", "inverse_filtered_cov3d",
                             "filtered_masses", "tiles_touched", "point_offsets", "i_ranges")]
    lst, cap = None, 0
    if want_list:
        P = L.orc_vr_forward_f32(*args, *outs, None, 0)
        lst = np.zeros(max(P, 1), np.uint32)
        cap = P
    P = L.orc_vr_forward_f32(*args, *outs, lst.ctypes.data if lst is not None else None, cap)
    out["n_pairs"] = P
    if want_list:
        out["point_list"] = lst[:P]
    return out


def vm_forward(scene, cam, bg=None, dtype=np.float32, cov_mult=1.0, render_mode=0, debug_bin=-1, max_depth=20.0):
    """vol_marcher forward.  Returns the reference's 13-entry cache as a dict
    (plus 'keys' and 'status').  render_mode: 0 Full, 1 Bins, 2 Depth."""
    L = lib()
    L.orc_set_render_mode(int(render_mode), int(debug_bin), float(max_depth))
    sfx = "f32" if dtype == np.float32 else "f64"
    N, W, H = scene.n, cam.width, cam.height
    gx, gy = tiles(cam)
    c = _vm_cache(N, W, H, gx, gy, dtype)
    args = _scene_args(scene, cam, dtype, bg, cov_mult)
    cl = [c[k] for k in _VM_ORDER]
    P = getattr(L, f"orc_vm_preprocess_{sfx}")(*args, *cl)
    c["b_point_list"] = np.zeros(max(P, 1), np.int32)
    keys = np.zeros(max(P, 1), np.uint64)
    c["status"] = getattr(L, f"orc_vm_render_{sfx}")(*args, *cl, c["b_point_list"], keys.ctypes.data)
    c["b_point_list"] = c["b_point_list"][:P]
    c["keys"] = keys[:P]
    c["n_pairs"] = P
    return c


def vm_backward(scene, cam, cache, grad_fb, bg=None, dtype=np.float32, cov_mult=1.0):
    L = lib()
    sfx = "f32" if dtype == np.float32 else "f64"
    N = scene.n
    k = scene.sh.shape[1]
    g = dict(sh=np.zeros((N, k, 3), dtype), weights=np.zeros(N, dtype), centroids=np.zeros((N, 3), dtype),
             scales=np.zeros((N, 3), dtype), rotations=np.zeros((N, 4), dtype))
    cl = [np.ascontiguousarray(cache[k]) for k in _VM_ORDER]
    lst = _c(cache["b_point_list"], np.int32)
    if lst.size == 0:
        lst = np.zeros(1, np.int32)
    st = getattr(L, f"orc_vm_backward_{sfx}")(*_scene_args(scene, cam, dtype, bg, cov_mult), *cl, lst,
                                                _c(grad_fb, dtype), g["sh"], g["weights"], g["centroids"],
                                                g["scales"], g["rotations"])
    g["status"] = st
    return g


def density_array(capacity, start, puts, dtype=np.float32):
    sfx = "f32" if dtype == np.float32 else "f64"
    ops = _c(np.asarray(puts, dtype=np.float64).reshape(-1, 3) if len(puts) else np.zeros((0, 3)), dtype).reshape(-1)
    if ops.size == 0:
        ops = np.zeros(3, dtype)
    out = np.zeros(16 * 3, dtype)
    end = np.zeros(1, dtype)
    n = getattr(lib(), f"orc_density_array_{sfx}")(capacity, start, ops, len(puts), out, end)
    return out[:3 * n].reshape(n, 3), float(end[0])


def density_combine(a, b, dtype=np.float32):
    sfx = "f32" if dtype == np.float32 else "f64"
    out = np.zeros(9, dtype)
    getattr(lib(), f"orc_density_combine_{sfx}")(_c(a, dtype), _c(b, dtype), out)
    return out.reshape(3, 3)


def density_sample(capacity, start, puts, n_samples, dtype=np.float32):
    sfx = "f32" if dtype == np.float32 else "f64"
    ops = _c(np.asarray(puts, dtype=np.float64).reshape(-1, 3) if len(puts) else np.zeros((0, 3)), dtype).reshape(-1)
    if ops.size == 0:
        ops = np.zeros(3, dtype)
    out = np.zeros(n_samples, dtype)
    getattr(lib(), f"orc_density_sample_{sfx}")(capacity, start, ops, len(puts), n_samples, out)
    return out


def fmath(which: str, x, libm: bool = False):
    """The shared fixed-sequence exp / log / erf (float) on x, or with
    ``libm`` the host C library's."""
    x = _c(x, np.float32)
    y = np.zeros_like(x)
    lib().orc_fmath_f32({"exp": 0, "log": 1, "erf": 2}[which] + (3 if libm else 0), x, y, x.size)
    return y


def pick2(which: str, v):
    """math.h:112-155 on float rows of 3: "larger" or "smaller" two components."""
    v = _c(np.asarray(v, np.float32).reshape(-1, 3), np.float32)
    out = np.zeros((v.shape[0], 2), np.float32)
    lib().orc_pick2_f32({"larger": 0, "smaller": 1}[which], v, out, v.shape[0])
    return out


@contextlib.contextmanager
def decision_audit():
    """Counts, inside the block, the float threshold decisions that depend on
    exp or log (splat alpha >= 1/255, ray-section mass >= 1/255, marcher
    rectangle radius) and how many of them the host libm's function would
    have taken the other way, and how many lie within 16 float ulps of the
    threshold (the only ones any exp / log within 16 ulps of the shared
    routines could flip).  Yields a dict filled on exit:
    {kind: (seen, flipped, near)}, plus "fills": the marcher's (ray,
    Gaussian, large step) bin fills of the block."""
    L = lib()
    out = np.zeros(10, np.int64)
    L.orc_audit(1, out.ctypes.data_as(C.POINTER(C.c_long)))
    res: dict = {}
    try:
        yield res
    finally:
        L.orc_audit(0, out.ctypes.data_as(C.POINTER(C.c_long)))
        for k, name in enumerate(("alpha", "section_mass", "rect")):
            res[name] = (int(out[3 * k]), int(out[3 * k + 1]), int(out[3 * k + 2]))
        res["fills"] = int(out[9])


def set_const_samples(sections) -> None:
    """Fix the marcher's sample sections, [(start, end, delta_t), ...]; [] restores adaptive sampling."""
    arr = np.ascontiguousarray(np.asarray(sections, dtype=np.float64).reshape(-1), dtype=np.float64)
    if arr.size == 0:
        arr = np.zeros(3)
    lib().orc_set_const_samples(len(sections), arr)


def density_randomised(iters=1000, puts=100, probes=50, dtype=np.float32) -> int:
    """The reference's srand(0) randomised DensityArray test; returns #failed checks."""
    sfx = "f32" if dtype == np.float32 else "f64"
    return int(getattr(lib(), f"orc_density_randomised_{sfx}")(iters, puts, probes))
