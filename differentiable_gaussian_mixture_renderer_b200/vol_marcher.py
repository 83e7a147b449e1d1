"""Differentiable volume ray marcher -- drop-in for python_bindings/vol_marcher.py.

``apply(shs, opacity, means3D, scales, rotations, world_view_transform,
full_proj_transform, camera_center, bg_color, image_width, image_height,
tanfovx, tanfovy, active_sh_degree) -> image [3, H, W]`` with the reference's
argument meaning (vol_marcher.py:19-65): float32 or float64 CUDA tensors,
matrices in the transposed (torch) layout, SH [N, k<=16, 3], opacity [N] or
[N, 1], rotations (w, x, y, z).  Backward returns gradients for the first five
inputs and None for the rest.  An optional 15th argument names the formulation
(opacity, mass, density, ots, ols; vol_marcher.h:66 fixes Opacity at compile
time, which None keeps).
"""
from __future__ import annotations

import torch

from . import _native as N
from . import cpp_binding

# The backward recomputes each ray's section sets and sample positions (as the
# reference does) only when memory is tight: a frame whose step store -- the
# first STORE_STEPS large steps of every ray -- takes at most
# STORE_MEMORY_FRACTION of the free device memory keeps them from the forward
# instead (same results, a shorter backward).  STORE_STEPS = 0 always recomputes.
STORE_STEPS = 4
STORE_MEMORY_FRACTION = 0.25


def _step_store(width: int, height: int, dtype, device):
    if STORE_STEPS <= 0:
        return None
    nbytes = N.lib().dgmr_vm_step_store_size(int(width), int(height), STORE_STEPS, N.dtype_code(dtype))
    free, _ = torch.cuda.mem_get_info(device)
    if nbytes == 0 or nbytes > free * STORE_MEMORY_FRACTION:
        return None
    return cpp_binding.make_step_store(width, height, STORE_STEPS, dtype, device)


class VolMarcher(torch.autograd.Function):
    @staticmethod
    def forward(ctx, shs, opacity, means3D, scales, rotations, world_view_transform, full_proj_transform,
                camera_center, bg_color, image_width: int, image_height: int, tanfovx: float, tanfovy: float,
                active_sh_degree: int, formulation: str | None = None):
        store = _step_store(image_width, image_height, means3D.dtype, means3D.device) \
            if any(ctx.needs_input_grad[:5]) else None
        cache = cpp_binding.forward(shs, opacity, means3D, scales, rotations, world_view_transform,
                                    full_proj_transform, camera_center, bg_color, image_width, image_height, tanfovx,
                                    tanfovy, active_sh_degree, formulation=formulation, step_store=store)
        ctx.step_store = store
        ctx.save_for_backward(shs, opacity, means3D, scales, rotations, world_view_transform, full_proj_transform,
                              camera_center, bg_color, *cache)
        ctx.frame = (int(image_width), int(image_height), float(tanfovx), float(tanfovy), int(active_sh_degree))
        ctx.formulation = formulation
        return cache[0]

    @staticmethod
    def backward(ctx, grad_output):
        if not grad_output.is_contiguous():
            grad_output = grad_output.contiguous()
        saved = ctx.saved_tensors
        shs, opacity, means3D, scales, rotations, view, proj, campos, bg = saved[:9]
        cache = list(saved[9:])
        W, H, tfx, tfy, deg = ctx.frame
        g_sh, g_w, g_mu, g_s, g_q = cpp_binding.backward(shs, opacity, means3D, scales, rotations, view, proj, campos,
                                                         bg, W, H, tfx, tfy, deg, grad_output, cache,
                                                         formulation=ctx.formulation, step_store=ctx.step_store)
        ctx.step_store = None
        if opacity.dim() == 1:
            g_w = g_w.reshape(-1)
        return g_sh, g_w, g_mu, g_s, g_q, None, None, None, None, None, None, None, None, None, None


apply = VolMarcher.apply
