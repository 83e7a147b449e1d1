"""The reference's torch extension surface, over the C ABI.

Mirrors ``cpp_binding.forward`` / ``cpp_binding.backward`` of
python_bindings/vol_marcher.cu:217-304: same argument order and meaning, same
13-entry cache (vol_marcher.cu:109-122), same gradient list.  Differences,
all deliberate:

* errors raise (TypeError / ValueError / DgmrError) instead of printing and
  returning an empty list (vol_marcher.cu:253-255);
* an empty frame (no visible Gaussian) renders the background and returns a
  valid cache with an empty point list, where the reference returns undefined
  cache tensors and a zero image (vol_marcher_forward.cu:194-195);
* SH coefficients are not concatenated to 16 on the device: the kernels read
  coefficients past the caller's count as 0 (forward) / 1 (backward), the
  values the reference pads with (vol_marcher.cu:92, :177).
"""
from __future__ import annotations

import numpy as np
import torch

from . import _native as N


def _f32(v: float) -> float:
    # the reference's binding takes tan_fov as C float (vol_marcher.cu:228-229)
    return float(np.float32(v))


def _check_inputs(tensors, names):
    dt = tensors[0].dtype
    for t, n in zip(tensors, names):
        if not isinstance(t, torch.Tensor):
            raise TypeError(f"{n} must be a torch.Tensor")
        if t.dtype != dt:
            raise TypeError("All input vectors must be of the same type (float32 or float64)")
    if dt not in (torch.float32, torch.float64):
        raise TypeError("All input vectors must be of the same type (float32 or float64)")
    dev = tensors[0].device
    if dev.type != "cuda":
        raise ValueError("vol_marcher runs on CUDA tensors only")
    for t, n in zip(tensors[:5], names[:5]):
        if t.device != dev:
            raise ValueError(f"{n} is on {t.device}, expected {dev}")
    return dt, dev


def _contig(t):
    return t if t.is_contiguous() else t.contiguous()


_MODES = {"full": N.RENDER_FULL, "bins": N.RENDER_BINS, "depth": N.RENDER_DEPTH}


def forward(sh_params, weights, centroids, cov_scales, cov_rotations, view_matrix, proj_matrix, cam_position,
            background, render_width: int, render_height: int, tan_fovx: float, tan_fovy: float, sh_degree: int,
            render_mode: str = "full", debug_render_bin: int = -1, max_depth: float = 20.0,
            formulation: str | None = None, work_counter: torch.Tensor | None = None, step_store=None):
    """``render_mode`` / ``debug_render_bin`` / ``max_depth`` are
    vol_marcher::ForwardData's debug fields (vol_marcher.h:48-56), which the
    reference's Python binding leaves at their defaults (Full, -1, 20).
    ``formulation`` (opacity, mass, density, ots, ols) replaces the compile-time
    vol_marcher::config::gaussian_mixture_formulation (vol_marcher.h:66); None
    keeps its Opacity.  backward must be given the same one.
    ``work_counter`` (an int64 device tensor of one element, not in the
    reference): the march adds its (ray, Gaussian, large step) bin fills to it.
    ``step_store`` (not in the reference): ``(uint8 device tensor, steps)``
    from ``make_step_store``; the forward keeps its sample steps there for a
    backward given the same store."""
    names = ("sh_params", "weights", "centroids", "cov_scales", "cov_rotations", "view_matrix", "proj_matrix",
             "cam_position", "background")
    dt, dev = _check_inputs([sh_params, weights, centroids, cov_scales, cov_rotations, view_matrix, proj_matrix,
                             cam_position, background], names)
    lib = N.lib()
    W, H = int(render_width), int(render_height)
    n = int(weights.shape[0])
    sh_params, weights, centroids = _contig(sh_params), _contig(weights), _contig(centroids)
    cov_scales, cov_rotations = _contig(cov_scales), _contig(cov_rotations)
    with torch.cuda.device(dev):
        scene = N.make_scene(sh_params, weights, centroids, cov_scales, cov_rotations, sh_degree, formulation)
        cam = N.make_camera(view_matrix, proj_matrix, cam_position, background, W, H, _f32(tan_fovx), _f32(tan_fovy))
        gx, gy = (W + 15) // 16, (H + 15) // 16
        opt = dict(device=dev)
        cache = [torch.empty((3, H, W), dtype=dt, **opt),
                 torch.empty((n, 2), dtype=torch.int32, **opt),
                 torch.empty((n, 3), dtype=dt, **opt),
                 torch.empty((n, 3), dtype=torch.bool, **opt),
                 torch.empty((n,), dtype=dt, **opt),
                 torch.empty((n, 2), dtype=dt, **opt),
                 torch.empty((n, 6), dtype=dt, **opt),
                 torch.empty((n,), dtype=dt, **opt),
                 torch.empty((n,), dtype=torch.int32, **opt),
                 torch.empty((n,), dtype=torch.int32, **opt),
                 torch.empty((gx * gy, 2), dtype=torch.int32, **opt),
                 None,
                 torch.empty((H, W), dtype=dt, **opt)]
        c = N.VmCache(*[N.ptr(t) for t in cache])
        stream = N.stream_handle()
        dcode = N.dtype_code(dt)
        ws_pre = torch.empty(lib.dgmr_vm_workspace_size(n, W, H, 0, dcode), dtype=torch.uint8, **opt)
        N.check(lib.dgmr_vm_forward_preprocess(scene, cam, c, N.ptr(ws_pre), ws_pre.numel(), None, stream),
                "vol_marcher forward preprocess")
        # the pair count sizes b_point_list, as in the reference (.item(), vol_marcher_forward.cu:193)
        n_pairs = int(cache[9][-1].item()) if n > 0 else 0
        cache[11] = torch.empty((n_pairs,), dtype=torch.int32, **opt)
        c.b_point_list = N.ptr(cache[11]) if n_pairs > 0 else None
        ws = torch.empty(lib.dgmr_vm_workspace_size(n, W, H, n_pairs, dcode), dtype=torch.uint8, **opt)
        if render_mode not in _MODES:
            raise ValueError(f"render_mode must be one of {sorted(_MODES)}")
        opts = N.RenderOptions(_MODES[render_mode], int(debug_render_bin), float(max_depth),
                               N.ptr(work_counter) if work_counter is not None else None)
        if step_store is None:
            N.check(lib.dgmr_vm_forward_render_options(scene, cam, opts, c, n_pairs, N.ptr(ws), ws.numel(), None, stream),
                    "vol_marcher forward render")
        else:
            buf, steps = step_store
            N.check(lib.dgmr_vm_forward_render_stored(scene, cam, opts, c, n_pairs, N.ptr(ws), ws.numel(), N.ptr(buf),
                                                      buf.numel(), int(steps), None, stream), "vol_marcher forward render")
    return cache


def backward(sh_params, weights, centroids, cov_scales, cov_rotations, view_matrix, proj_matrix, cam_position,
             background, render_width: int, render_height: int, tan_fovx: float, tan_fovy: float, sh_degree: int,
             grad_framebuffer, cache_vector, formulation: str | None = None, step_store=None):
    names = ("sh_params", "weights", "centroids", "cov_scales", "cov_rotations", "view_matrix", "proj_matrix",
             "cam_position", "background")
    dt, dev = _check_inputs([sh_params, weights, centroids, cov_scales, cov_rotations, view_matrix, proj_matrix,
                             cam_position, background], names)
    if grad_framebuffer.dtype != dt:
        raise TypeError("grad_framebuffer must have the inputs' dtype")
    lib = N.lib()
    W, H = int(render_width), int(render_height)
    n = int(weights.shape[0])
    sh_params, weights, centroids = _contig(sh_params), _contig(weights), _contig(centroids)
    cov_scales, cov_rotations = _contig(cov_scales), _contig(cov_rotations)
    grad_framebuffer = _contig(grad_framebuffer)
    cache = [_contig(t) if t is not None else None for t in cache_vector]
    with torch.cuda.device(dev):
        scene = N.make_scene(sh_params, weights, centroids, cov_scales, cov_rotations, sh_degree, formulation)
        cam = N.make_camera(view_matrix, proj_matrix, cam_position, background, W, H, _f32(tan_fovx), _f32(tan_fovy))
        opt = dict(device=dev, dtype=dt)
        k = int(sh_params.shape[1])
        g_sh = torch.empty((n, k, 3), **opt)
        g_w = torch.empty((n, 1), **opt)
        g_mu = torch.empty((n, 3), **opt)
        g_s = torch.empty((n, 3), **opt)
        g_q = torch.empty((n, 4), **opt)
        c = N.VmCache(*[N.ptr(t) if (t is not None and t.numel() > 0) else None for t in cache])
        if c.b_point_list is None:
            c.b_point_list = N.ptr(cache[9])  # never read: the tile ranges are all empty
        # sized with the frame's pair count: the march uses the room for its per-ray Gaussian masks
        n_pairs = int(cache[11].numel()) if cache[11] is not None else 0
        ws = torch.empty(lib.dgmr_vm_workspace_size(n, W, H, n_pairs, N.dtype_code(dt)), dtype=torch.uint8, device=dev)
        if step_store is None:
            N.check(lib.dgmr_vm_backward(scene, cam, c, N.ptr(grad_framebuffer), N.ptr(g_sh), N.ptr(g_w), N.ptr(g_mu),
                                         N.ptr(g_s), N.ptr(g_q), N.ptr(ws), ws.numel(), None, N.stream_handle()),
                    "vol_marcher backward")
        else:
            buf, steps = step_store
            N.check(lib.dgmr_vm_backward_stored(scene, cam, c, N.ptr(grad_framebuffer), N.ptr(g_sh), N.ptr(g_w),
                                                N.ptr(g_mu), N.ptr(g_s), N.ptr(g_q), N.ptr(ws), ws.numel(), N.ptr(buf),
                                                buf.numel(), int(steps), None, N.stream_handle()), "vol_marcher backward")
    return [g_sh, g_w, g_mu, g_s, g_q]


def make_step_store(render_width: int, render_height: int, steps: int, dtype=torch.float32, device=None):
    """A sample-step store for ``steps`` large steps of every ray of a frame
    (not in the reference): pass it to forward and to the backward of the
    same frame, which then skips recomputing those steps' section sets and
    sample positions.  Returns ``(tensor, steps)``."""
    lib = N.lib()
    nbytes = lib.dgmr_vm_step_store_size(int(render_width), int(render_height), int(steps), N.dtype_code(dtype))
    if nbytes == 0:
        raise ValueError("invalid step store size")
    return torch.empty(nbytes, dtype=torch.uint8, device=device or "cuda"), int(steps)


def set_const_samples(sections) -> None:
    """Gradient-check mode (the reference's DGMR_TORCH_GRAD_CHECK_CONST_SAMPLES):
    fixed (start, end, delta_t) sample sections; [] restores adaptive sampling."""
    arr = np.ascontiguousarray(np.asarray(sections, dtype=np.float64).reshape(-1))
    lib = N.load()
    N.check(lib.dgmr_vm_set_const_samples(len(sections), arr.ctypes.data if arr.size else None),
            "set_const_samples")
