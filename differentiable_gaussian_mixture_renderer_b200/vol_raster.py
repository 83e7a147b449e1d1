"""Volume rasteriser (the reference's dgmr::vol_raster_forward,
src/dgmr/vol_raster_forward.cu:39-520): forward-only, float32.

Inputs are the reference's layouts (the same as the vol_marcher binding's):
sh [N,k,3], weights [N] or [N,1], centroids [N,3], scales [N,3], rotations
[N,4] (w,x,y,z), view / proj as the torch tensors whose row-major bytes are the
glm matrices, campos [3], background [3].
"""
from __future__ import annotations

import torch

from . import _native as N

_MODES = {"full": N.RENDER_FULL, "bins": N.RENDER_BINS, "depth": N.RENDER_DEPTH}


def forward(sh, weights, centroids, scales, rotations, view, proj, campos, background, width: int, height: int,
            tan_fovx: float, tan_fovy: float, sh_degree: int, cov_scale_multiplier: float = 1.0,
            render_mode: str = "full", debug_bin: int = -1, max_depth: float = 20.0,
            stream: torch.cuda.Stream | None = None, formulation: str | None = None) -> torch.Tensor:
    """Render one frame; returns the framebuffer [3, H, W].  The pair buffers are
    sized from the frame (preprocess, pair count read back, then the render),
    like the reference's .item() read of the pair count.  ``formulation``
    (opacity, mass, density, ots, ols) replaces the compile-time
    vol_raster::config::gaussian_mixture_formulation (vol_raster_forward.h:66);
    None keeps its Ots."""
    ts = [sh, weights, centroids, scales, rotations]
    for t in ts:
        if not isinstance(t, torch.Tensor) or t.dtype != torch.float32:
            raise TypeError("vol_raster takes float32 tensors")
        if t.device.type != "cuda":
            raise ValueError("vol_raster runs on CUDA tensors only")
    if render_mode not in _MODES:
        raise ValueError(f"render_mode must be one of {sorted(_MODES)}")
    sh, weights, centroids, scales, rotations = [t if t.is_contiguous() else t.contiguous() for t in ts]
    lib = N.lib()
    dev = centroids.device
    n, W, H = int(centroids.shape[0]), int(width), int(height)
    with torch.cuda.device(dev):
        scene = N.make_scene(sh, weights, centroids, scales, rotations, sh_degree, formulation)
        cam = N.make_camera(view, proj, campos, background, W, H, tan_fovx, tan_fovy, cov_scale_multiplier)
        opts = N.RenderOptions(_MODES[render_mode], int(debug_bin), float(max_depth))
        s = N.stream_handle(stream)
        stats = torch.zeros(4, dtype=torch.int32, device=dev)
        frame_ws = torch.empty(max(1, lib.dgmr_vr_frame_workspace_size(n, W, H)), dtype=torch.uint8, device=dev)
        N.check(lib.dgmr_vr_preprocess(scene, cam, N.ptr(frame_ws), frame_ws.numel(), N.ptr(stats), s),
                "vol_raster preprocess")
        cap = int(stats[0].item())
        pair_ws = torch.empty(max(1, lib.dgmr_vr_pair_workspace_size(n, cap)), dtype=torch.uint8, device=dev)
        fb = torch.empty((3, H, W), dtype=torch.float32, device=dev)
        N.check(lib.dgmr_vr_forward(scene, cam, opts, N.ptr(fb), N.ptr(frame_ws), frame_ws.numel(), N.ptr(pair_ws),
                                    pair_ws.numel(), cap, N.ptr(stats), s), "vol_raster forward")
    return fb
