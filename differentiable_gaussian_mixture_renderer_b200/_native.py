"""ctypes view of libdgmr_b200.so (declarations in include/dgmr_b200.h).

The product path has no CPU fallback: if the library or a CUDA device is
missing, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os

import torch

from . import build as _build

DGMR_OK, DGMR_ERR_BAD_ARG, DGMR_ERR_WORKSPACE, DGMR_ERR_CUDA, DGMR_ERR_STATIC_SCRATCH = 0, 1, 2, 3, 4
DGMR_ERR_PAIR_OVERFLOW = 5
DGMR_F32, DGMR_F64 = 0, 1
FLAG_PAIR_OVERFLOW, FLAG_STEP_LIMIT = 1, 2


class DgmrError(RuntimeError):
    pass


class Scene(C.Structure):
    _fields_ = [("n_gaussians", C.c_int32), ("sh_stride", C.c_int32), ("sh_degree", C.c_int32), ("dtype", C.c_int32),
                ("centroids", C.c_void_p), ("sh", C.c_void_p), ("weights", C.c_void_p), ("scales", C.c_void_p),
                ("rotations", C.c_void_p), ("formulation", C.c_int32), ("reserved", C.c_int32)]


# dgmr_formulation codes (types.h:26-32 plus 1; 0 keeps each renderer's reference default)
FORMULATIONS = {None: 0, "opacity": 1, "mass": 2, "density": 3, "ots": 4, "ols": 5}


def formulation_code(f) -> int:
    """Maps a formulation name (or None for the renderer's default, or a code)
    to its dgmr_formulation value; raises ValueError for anything else."""
    if isinstance(f, int) and not isinstance(f, bool):
        if 0 <= f <= 5:
            return f
    elif f is None or isinstance(f, str):
        key = f.lower() if isinstance(f, str) else f
        if key in FORMULATIONS:
            return FORMULATIONS[key]
    raise ValueError(f"unknown formulation {f!r}: one of opacity, mass, density, ots, ols")


class Camera(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("view", C.c_double * 16), ("proj", C.c_double * 16),
                ("campos", C.c_double * 3), ("background", C.c_double * 3), ("tan_fovx", C.c_double),
                ("tan_fovy", C.c_double), ("cov_scale_multiplier", C.c_double)]


class FrameStats(C.Structure):
    _fields_ = [("n_pairs", C.c_uint32), ("flags", C.c_uint32), ("n_visible", C.c_uint32), ("reserved", C.c_uint32)]


_VM_CACHE_FIELDS = ("framebuffer", "rects", "rgb", "rgb_sh_clamped", "depths", "points_xy_image",
                    "inverse_filtered_cov3d", "filtered_masses", "tiles_touched", "point_offsets", "i_ranges",
                    "b_point_list", "remaining_transparency")


class VmCache(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in _VM_CACHE_FIELDS]


_SPLAT_VIEW_FIELDS = ("rects", "rgb", "rgb_sh_clamped", "depths", "points_xy_image", "conic_opacity", "tiles_touched",
                      "point_offsets", "i_ranges", "point_list", "point_list_tiles", "final_transmittance",
                      "n_contrib")


class SplatViews(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in _SPLAT_VIEW_FIELDS]


BATCH_MAX_VIEWS, BATCH_MAX_SCENES = 64, 16


class BatchView(C.Structure):
    _fields_ = [("scene", C.c_int32), ("blend_block", C.c_int32), ("camera", Camera), ("framebuffer", C.c_void_p),
                ("grad_framebuffer", C.c_void_p)]


class SceneGrads(C.Structure):
    _fields_ = [("sh", C.c_void_p), ("weights", C.c_void_p), ("centroids", C.c_void_p), ("scales", C.c_void_p),
                ("rotations", C.c_void_p)]


SERVE_SPLAT, SERVE_MARCH = 0, 1


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("n_slots", C.c_int32), ("max_views", C.c_int32), ("reserved", C.c_int32),
                ("hbm_budget_bytes", C.c_size_t), ("capacity_margin", C.c_double), ("max_batch_pixels", C.c_int64)]


class ServerRequest(C.Structure):
    _fields_ = [("kind", C.c_int32), ("scene", C.c_int32), ("camera", Camera), ("framebuffer", C.c_void_p),
                ("grad_image", C.c_void_p), ("grads", SceneGrads), ("host_image", C.c_void_p), ("tag", C.c_uint64)]


class ServerCompletion(C.Structure):
    _fields_ = [("tag", C.c_uint64), ("status", C.c_int), ("n_pairs", C.c_uint32), ("batch_size", C.c_int32),
                ("rerendered", C.c_int32), ("submit_s", C.c_double), ("launch_s", C.c_double), ("done_s", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_int64), ("batches", C.c_int64), ("rerenders", C.c_int64), ("deferred", C.c_int64),
                ("reallocs", C.c_int32), ("reserved", C.c_int32), ("hbm_budget_bytes", C.c_size_t),
                ("hbm_in_use_bytes", C.c_size_t), ("hbm_peak_bytes", C.c_size_t)]


RENDER_FULL, RENDER_BINS, RENDER_DEPTH = 0, 1, 2


class RenderOptions(C.Structure):
    _fields_ = [("render_mode", C.c_int32), ("debug_bin", C.c_int32), ("max_depth", C.c_double),
                ("work_counter", C.c_void_p)]


# every symbol include/dgmr_b200.h declares, with its ctypes signature
_SIGNATURES = {
    "dgmr_splat_frame_workspace_size": (C.c_size_t, [C.c_int32, C.c_int32, C.c_int32]),
    "dgmr_splat_pair_workspace_size": (C.c_size_t, [C.c_int32, C.c_int64]),
    "dgmr_splat_forward": (C.c_int, [C.POINTER(Scene), C.POINTER(Camera), C.c_void_p, C.c_void_p, C.c_size_t,
                                     C.c_void_p, C.c_size_t, C.c_int64, C.c_void_p, C.c_void_p]),
    "dgmr_splat_preprocess": (C.c_int, [C.POINTER(Scene), C.POINTER(Camera), C.c_void_p, C.c_size_t, C.c_void_p,
                                        C.c_void_p]),
    "dgmr_splat_render": (C.c_int, [C.POINTER(Scene), C.POINTER(Camera), C.c_void_p, C.c_void_p, C.c_size_t,
                                    C.c_void_p, C.c_size_t, C.c_int64, C.c_void_p, C.c_void_p]),
    "dgmr_splat_workspace_views": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, C.c_int64, C.c_void_p, C.c_size_t,
                                             C.c_void_p, C.c_size_t, C.POINTER(SplatViews)]),
    "dgmr_splat_blend": (C.c_int, [C.POINTER(Camera), C.c_int32, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p,
                                   C.c_size_t, C.c_int64, C.c_void_p]),
    "dgmr_splat_forward_noalloc": (C.c_int, [C.POINTER(Scene), C.POINTER(Camera), C.c_void_p, C.c_int64, C.c_void_p,
                                             C.c_void_p]),
    "dgmr_splat_backward": (C.c_int, [C.POINTER(Scene), C.POINTER(Camera), C.c_void_p, C.c_void_p, C.c_void_p,
                                      C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p,
                                      C.c_size_t, C.c_int64, C.c_void_p]),
    "dgmr_splat_batch_workspace_size": (C.c_int, [C.POINTER(Scene), C.c_int32, C.POINTER(BatchView), C.c_int32,
                                                  C.c_int64, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "dgmr_splat_batch_preprocess": (C.c_int, [C.POINTER(Scene), C.c_int32, C.POINTER(BatchView), C.c_int32,
                                              C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p]),
    "dgmr_splat_batch_forward": (C.c_int, [C.POINTER(Scene), C.c_int32, C.POINTER(BatchView), C.c_int32, C.c_void_p,
                                           C.c_size_t, C.c_void_p, C.c_size_t, C.c_int64, C.c_void_p, C.c_void_p]),
    "dgmr_splat_batch_backward": (C.c_int, [C.POINTER(Scene), C.c_int32, C.POINTER(BatchView), C.c_int32,
                                            C.POINTER(SceneGrads), C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t,
                                            C.c_int64, C.c_void_p]),
    "dgmr_vm_batch_workspace_size": (C.c_int, [C.POINTER(Scene), C.c_int32, C.POINTER(BatchView), C.c_int32,
                                               C.c_int64, C.POINTER(C.c_size_t), C.POINTER(C.c_size_t)]),
    "dgmr_vm_batch_preprocess": (C.c_int, [C.POINTER(Scene), C.c_int32, C.POINTER(BatchView), C.c_int32,
                                           C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p]),
    "dgmr_vm_batch_forward": (C.c_int, [C.POINTER(Scene), C.c_int32, C.POINTER(BatchView), C.c_int32, C.c_void_p,
                                        C.c_size_t, C.c_void_p, C.c_size_t, C.c_int64, C.c_void_p, C.c_void_p]),
    "dgmr_vm_batch_backward": (C.c_int, [C.POINTER(Scene), C.c_int32, C.POINTER(BatchView), C.c_int32,
                                         C.POINTER(SceneGrads), C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t,
                                         C.c_int64, C.c_void_p, C.c_void_p]),
    "dgmr_batch_autotune": (C.c_int, [C.c_int32, C.POINTER(Scene), C.c_int32, C.POINTER(BatchView), C.c_int32,
                                      C.POINTER(SceneGrads), C.POINTER(C.c_int32), C.c_int32, C.POINTER(C.c_int32),
                                      C.c_int32, C.c_int32, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_int64,
                                      C.POINTER(C.c_float), C.POINTER(C.c_int32), C.POINTER(C.c_int32), C.c_void_p]),
    "dgmr_vr_frame_workspace_size": (C.c_size_t, [C.c_int32, C.c_int32, C.c_int32]),
    "dgmr_vr_pair_workspace_size": (C.c_size_t, [C.c_int32, C.c_int64]),
    "dgmr_vr_preprocess": (C.c_int, [C.POINTER(Scene), C.POINTER(Camera), C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p]),
    "dgmr_vr_forward": (C.c_int, [C.POINTER(Scene), C.POINTER(Camera), C.POINTER(RenderOptions), C.c_void_p, C.c_void_p, C.c_size_t,
                                  C.c_void_p, C.c_size_t, C.c_int64, C.c_void_p, C.c_void_p]),
    "dgmr_vm_workspace_size": (C.c_size_t, [C.c_int32, C.c_int32, C.c_int32, C.c_int64, C.c_int32]),
    "dgmr_vm_forward_preprocess": (C.c_int, [C.POINTER(Scene), C.POINTER(Camera), C.POINTER(VmCache), C.c_void_p,
                                             C.c_size_t, C.c_void_p, C.c_void_p]),
    "dgmr_vm_forward_render": (C.c_int, [C.POINTER(Scene), C.POINTER(Camera), C.POINTER(VmCache), C.c_int64,
                                         C.c_void_p, C.c_size_t, C.c_void_p, C.c_void_p]),
    "dgmr_vm_forward_render_options": (C.c_int, [C.POINTER(Scene), C.POINTER(Camera), C.POINTER(RenderOptions),
                                                 C.POINTER(VmCache), C.c_int64, C.c_void_p, C.c_size_t, C.c_void_p,
                                                 C.c_void_p]),
    "dgmr_vm_backward": (C.c_int, [C.POINTER(Scene), C.POINTER(Camera), C.POINTER(VmCache), C.c_void_p, C.c_void_p,
                                   C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t,
                                   C.c_void_p, C.c_void_p]),
    "dgmr_vm_step_store_size": (C.c_size_t, [C.c_int32, C.c_int32, C.c_int32, C.c_int32]),
    "dgmr_vm_forward_render_stored": (C.c_int, [C.POINTER(Scene), C.POINTER(Camera), C.POINTER(RenderOptions),
                                                C.POINTER(VmCache), C.c_int64, C.c_void_p, C.c_size_t, C.c_void_p,
                                                C.c_size_t, C.c_int32, C.c_void_p, C.c_void_p]),
    "dgmr_vm_backward_stored": (C.c_int, [C.POINTER(Scene), C.POINTER(Camera), C.POINTER(VmCache), C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                          C.c_size_t, C.c_void_p, C.c_size_t, C.c_int32, C.c_void_p, C.c_void_p]),
    "dgmr_vm_set_const_samples": (C.c_int, [C.c_int32, C.c_void_p]),
    "dgmr_server_create": (C.c_int, [C.POINTER(ServerConfig), C.POINTER(C.c_void_p)]),
    "dgmr_server_add_scene": (C.c_int, [C.c_void_p, C.POINTER(Scene), C.POINTER(C.c_int32)]),
    "dgmr_server_submit": (C.c_int, [C.c_void_p, C.POINTER(ServerRequest)]),
    "dgmr_server_poll": (C.c_int32, [C.c_void_p, C.POINTER(ServerCompletion), C.c_int32]),
    "dgmr_server_wait": (C.c_int32, [C.c_void_p, C.POINTER(ServerCompletion), C.c_int32]),
    "dgmr_server_pending": (C.c_int64, [C.c_void_p]),
    "dgmr_server_now": (C.c_double, [C.c_void_p]),
    "dgmr_server_get_stats": (C.c_int, [C.c_void_p, C.POINTER(ServerStats)]),
    "dgmr_server_destroy": (C.c_int, [C.c_void_p]),
    "dgmr_status_string": (C.c_char_p, [C.c_int]),
    "dgmr_version": (C.c_char_p, []),
    "dgmr_launch_count": (C.c_uint64, []),
}

_lib = None


def library_path() -> str:
    return _build.LIB_PATH


def load(allow_build: bool = True):
    """Load (building first if needed and possible) and declare the library."""
    global _lib
    if _lib is not None:
        return _lib
    path = _build.LIB_PATH
    if not os.path.exists(path):
        if not allow_build:
            raise DgmrError(f"libdgmr_b200.so not found at {path}; build it with "
                            "python -m differentiable_gaussian_mixture_renderer_b200.build")
        _build.build()
    lib = C.CDLL(path)
    for name, (res, args) in _SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def lib():
    if _lib is None:
        if not torch.cuda.is_available():
            raise DgmrError("libdgmr_b200 needs a CUDA device; there is no CPU fallback")
        load()
    return _lib


def check(status: int, what: str) -> None:
    if status != DGMR_OK:
        msg = _lib.dgmr_status_string(status).decode() if _lib else str(status)
        raise DgmrError(f"{what} failed: {msg} (status {status})")


def ptr(t) -> int | None:
    return None if t is None else t.data_ptr()


def stream_handle(stream: torch.cuda.Stream | None = None) -> int:
    s = stream if stream is not None else torch.cuda.current_stream()
    return s.cuda_stream


def dtype_code(dtype: torch.dtype) -> int:
    if dtype == torch.float32:
        return DGMR_F32
    if dtype == torch.float64:
        return DGMR_F64
    raise TypeError("All input tensors must be of the same type (float32 or float64)")


def make_scene(shs, weights, centroids, scales, rotations, sh_degree: int, formulation=None) -> Scene:
    s = Scene()
    s.formulation = formulation_code(formulation)
    s.n_gaussians = int(centroids.shape[0])
    s.sh_stride = int(shs.shape[1])
    s.sh_degree = int(sh_degree)
    s.dtype = dtype_code(centroids.dtype)
    s.centroids, s.sh, s.weights = centroids.data_ptr(), shs.data_ptr(), weights.data_ptr()
    s.scales, s.rotations = scales.data_ptr(), rotations.data_ptr()
    return s


def _host_values(t, n: int) -> list[float]:
    if isinstance(t, torch.Tensor):
        return [float(v) for v in t.detach().reshape(-1)[:n].cpu().double().tolist()]
    import numpy as np
    return [float(v) for v in np.asarray(t, dtype=np.float64).reshape(-1)[:n]]


def make_camera(view, proj, campos, background, width: int, height: int, tan_fovx: float, tan_fovy: float,
                cov_scale_multiplier: float = 1.0) -> Camera:
    """view/proj in the torch layout of the reference (row i = glm column i)."""
    c = Camera()
    c.width, c.height = int(width), int(height)
    v = _host_values(view, 16)
    p = _host_values(proj, 16)
    for i in range(16):
        c.view[i] = v[i]
        c.proj[i] = p[i]
    cp = _host_values(campos, 3)
    bg = _host_values(background, 3)
    for i in range(3):
        c.campos[i] = cp[i]
        c.background[i] = bg[i]
    c.tan_fovx, c.tan_fovy = float(tan_fovx), float(tan_fovy)
    c.cov_scale_multiplier = float(cov_scale_multiplier)
    return c
