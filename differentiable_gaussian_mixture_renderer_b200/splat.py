"""Tile-based splat renderer: forward (the reference's dgmr::splat_forward,
src/dgmr/splat_forward.cu) and backward (new; the reference has none), as a
plain call and as a torch.autograd.Function.

Arguments follow the vol_marcher op's conventions: float32 CUDA tensors,
sh [N, k<=16, 3], opacity [N] or [N, 1], means [N, 3], scales [N, 3],
rotations [N, 4] (w, x, y, z), view / full view-projection matrices in the
transposed torch layout, background [3].
"""
from __future__ import annotations

from dataclasses import dataclass

import torch

from . import _native as N


@dataclass
class SplatFrame:
    """Device state of one rendered frame (kept for the backward pass)."""
    frame_ws: torch.Tensor
    pair_ws: torch.Tensor
    pair_capacity: int
    stats: torch.Tensor  # int32[4]: n_pairs, flags, ...
    scene: N.Scene
    camera: N.Camera
    n: int
    width: int
    height: int

    def ws_args(self):
        return (N.ptr(self.frame_ws), self.frame_ws.numel(), N.ptr(self.pair_ws), self.pair_ws.numel())

    def views(self) -> dict:
        """Per-Gaussian cache and binning result as tensors (no copies)."""
        lib = N.lib()
        v = N.SplatViews()
        N.check(lib.dgmr_splat_workspace_views(self.n, self.width, self.height, self.pair_capacity, *self.ws_args(), v),
                "workspace views")
        gx, gy = (self.width + 15) // 16, (self.height + 15) // 16
        n, hw, cap = self.n, self.width * self.height, self.pair_capacity

        def view(addr, count, dtype, shape):
            buf = self.frame_ws if self.frame_ws.data_ptr() <= addr < self.frame_ws.data_ptr() + self.frame_ws.numel() \
                else self.pair_ws
            elem = torch.tensor([], dtype=dtype).element_size()
            off = addr - buf.data_ptr()
            return buf[off:off + count * elem].view(dtype).reshape(shape)

        return dict(rects=view(v.rects, 2 * n, torch.int32, (n, 2)), rgb=view(v.rgb, 3 * n, torch.float32, (n, 3)),
                    rgb_sh_clamped=view(v.rgb_sh_clamped, 3 * n, torch.uint8, (n, 3)),
                    depths=view(v.depths, n, torch.float32, (n,)),
                    points_xy_image=view(v.points_xy_image, 2 * n, torch.float32, (n, 2)),
                    conic_opacity=view(v.conic_opacity, 4 * n, torch.float32, (n, 4)),
                    tiles_touched=view(v.tiles_touched, n, torch.int32, (n,)),
                    point_offsets=view(v.point_offsets, n, torch.int32, (n,)),
                    i_ranges=view(v.i_ranges, 2 * gx * gy, torch.int32, (gx * gy, 2)),
                    point_list=view(v.point_list, cap, torch.int32, (cap,)),
                    point_list_tiles=view(v.point_list_tiles, cap, torch.int32, (cap,)),
                    final_transmittance=view(v.final_transmittance, hw, torch.float32, (self.height, self.width)),
                    n_contrib=view(v.n_contrib, hw, torch.int32, (self.height, self.width)))


def _prepare(shs, opacity, means3D, scales, rotations):
    ts = [shs, opacity, means3D, scales, rotations]
    for t in ts:
        if not isinstance(t, torch.Tensor) or t.dtype != torch.float32:
            raise TypeError("the splat renderer takes float32 tensors")
        if t.device.type != "cuda":
            raise ValueError("the splat renderer runs on CUDA tensors only")
    return [t if t.is_contiguous() else t.contiguous() for t in ts]


def splat_forward(shs, opacity, means3D, scales, rotations, view, proj, campos, background, width: int, height: int,
                  tanfovx: float, tanfovy: float, sh_degree: int, cov_scale_multiplier: float = 1.0,
                  pair_capacity: int | None = None, framebuffer: torch.Tensor | None = None,
                  stream: torch.cuda.Stream | None = None, formulation: str | None = None
                  ) -> tuple[torch.Tensor, SplatFrame]:
    """Render one frame.

    Without ``pair_capacity`` the pair buffers are sized from the frame itself:
    preprocess, one device->host read of the pair count (the reference's
    .item() at splat_forward.cu:204), then binning and blend.  With it the call
    is asynchronous end to end; ``frame.stats[1] & 1`` then reports a frame
    that needed more pairs than the capacity.

    ``formulation`` picks how a weight becomes a screen-space opacity
    (math.h:322-380: opacity, mass, density, ots, ols); None keeps the splat
    renderer's Ots (splat_forward.h:58).  The backward of the frame uses the
    same one."""
    shs, opacity, means3D, scales, rotations = _prepare(shs, opacity, means3D, scales, rotations)
    lib = N.lib()
    dev = means3D.device
    n, W, H = int(means3D.shape[0]), int(width), int(height)
    scene = N.make_scene(shs, opacity, means3D, scales, rotations, sh_degree, formulation)
    cam = N.make_camera(view, proj, campos, background, W, H, tanfovx, tanfovy, cov_scale_multiplier)
    fb = framebuffer if framebuffer is not None else torch.empty((3, H, W), dtype=torch.float32, device=dev)
    stats = torch.zeros(4, dtype=torch.int32, device=dev)
    sh = N.stream_handle(stream)
    frame_ws = torch.empty(lib.dgmr_splat_frame_workspace_size(n, W, H), dtype=torch.uint8, device=dev)
    if pair_capacity is None:
        N.check(lib.dgmr_splat_preprocess(scene, cam, N.ptr(frame_ws), frame_ws.numel(), N.ptr(stats), sh),
                "splat preprocess")
        cap = int(stats[0].item())
        pair_ws = torch.empty(max(1, lib.dgmr_splat_pair_workspace_size(n, cap)), dtype=torch.uint8, device=dev)
        N.check(lib.dgmr_splat_render(scene, cam, N.ptr(fb), N.ptr(frame_ws), frame_ws.numel(), N.ptr(pair_ws),
                                      pair_ws.numel(), cap, N.ptr(stats), sh), "splat render")
    else:
        cap = int(pair_capacity)
        pair_ws = torch.empty(max(1, lib.dgmr_splat_pair_workspace_size(n, cap)), dtype=torch.uint8, device=dev)
        N.check(lib.dgmr_splat_forward(scene, cam, N.ptr(fb), N.ptr(frame_ws), frame_ws.numel(), N.ptr(pair_ws),
                                       pair_ws.numel(), cap, N.ptr(stats), sh), "splat forward")
    return fb, SplatFrame(frame_ws, pair_ws, cap, stats, scene, cam, n, W, H)


def splat_backward(frame: SplatFrame, grad_framebuffer: torch.Tensor, shs, opacity, means3D, scales, rotations,
                   stream: torch.cuda.Stream | None = None):
    """Gradients w.r.t. (shs, opacity, means3D, scales, rotations) of a frame
    rendered by splat_forward with the same tensors."""
    shs, opacity, means3D, scales, rotations = _prepare(shs, opacity, means3D, scales, rotations)
    lib = N.lib()
    g = grad_framebuffer if grad_framebuffer.is_contiguous() else grad_framebuffer.contiguous()
    if g.dtype != torch.float32 or tuple(g.shape) != (3, frame.height, frame.width):
        raise ValueError("grad_framebuffer must be float32 [3, H, W]")
    dev = means3D.device
    n = frame.n
    g_sh = torch.empty(shs.shape, dtype=torch.float32, device=dev)
    g_w = torch.empty(opacity.shape, dtype=torch.float32, device=dev)
    g_mu = torch.empty((n, 3), dtype=torch.float32, device=dev)
    g_s = torch.empty((n, 3), dtype=torch.float32, device=dev)
    g_q = torch.empty((n, 4), dtype=torch.float32, device=dev)
    N.check(lib.dgmr_splat_backward(frame.scene, frame.camera, N.ptr(g), N.ptr(g_sh), N.ptr(g_w), N.ptr(g_mu),
                                    N.ptr(g_s), N.ptr(g_q), *frame.ws_args(), frame.pair_capacity,
                                    N.stream_handle(stream)), "splat backward")
    return g_sh, g_w, g_mu, g_s, g_q


class SplatRender(torch.autograd.Function):
    @staticmethod
    def forward(ctx, shs, opacity, means3D, scales, rotations, view, proj, campos, background, width: int,
                height: int, tanfovx: float, tanfovy: float, sh_degree: int, formulation: str | None = None):
        fb, frame = splat_forward(shs, opacity, means3D, scales, rotations, view, proj, campos, background, width,
                                  height, tanfovx, tanfovy, sh_degree, formulation=formulation)
        ctx.frame = frame
        ctx.save_for_backward(shs, opacity, means3D, scales, rotations)
        return fb

    @staticmethod
    def backward(ctx, grad_output):
        shs, opacity, means3D, scales, rotations = ctx.saved_tensors
        grads = splat_backward(ctx.frame, grad_output, shs, opacity, means3D, scales, rotations)
        return (*grads, None, None, None, None, None, None, None, None, None, None)


render = SplatRender.apply


class SplatContext:
    """The plain per-call splat path with its workspaces kept between calls.

    Each ``forward`` is the reference's calling pattern
    (splat_forward.cu:41-338): preprocess, one read back of the pair count
    (its ``.item()`` at :204), binning and blend, one frame at a time on one
    stream.  The frame and pair workspaces grow when a frame needs more (with
    25 % headroom) and are never freed in between, as the C++ viewer
    interface's Context does, so steady calls allocate nothing."""

    def __init__(self, device=None, stream: torch.cuda.Stream | None = None, headroom: float = 1.25):
        self.device = torch.device(device or "cuda")
        self.stream = stream or torch.cuda.current_stream(self.device)
        self.headroom = headroom
        self.frame_ws = torch.empty(0, dtype=torch.uint8, device=self.device)
        self.pair_ws = torch.empty(0, dtype=torch.uint8, device=self.device)
        self.stats = torch.zeros(4, dtype=torch.int32, device=self.device)
        self.stats_host = torch.zeros(4, dtype=torch.int32, pin_memory=True)

    def _grow(self, buf: torch.Tensor, nbytes: int) -> torch.Tensor:
        if buf.numel() >= nbytes:
            return buf
        with torch.cuda.stream(self.stream):
            return torch.empty(int(nbytes * self.headroom) + 256, dtype=torch.uint8, device=self.device)

    def forward(self, shs, opacity, means3D, scales, rotations, camera: N.Camera, framebuffer: torch.Tensor,
                sh_degree: int, formulation: str | None = None) -> int:
        """Renders into ``framebuffer`` (float32 [3, H, W] on the device) and
        returns the frame's pair count; the call returns once the pair count
        is known, the image is complete when the stream reaches it."""
        shs, opacity, means3D, scales, rotations = _prepare(shs, opacity, means3D, scales, rotations)
        lib = N.lib()
        n, W, H = int(means3D.shape[0]), int(camera.width), int(camera.height)
        scene = N.make_scene(shs, opacity, means3D, scales, rotations, sh_degree, formulation)
        s = self.stream.cuda_stream
        self.frame_ws = self._grow(self.frame_ws, lib.dgmr_splat_frame_workspace_size(n, W, H))
        N.check(lib.dgmr_splat_preprocess(scene, camera, N.ptr(self.frame_ws), self.frame_ws.numel(), N.ptr(self.stats),
                                          s), "splat preprocess")
        with torch.cuda.stream(self.stream):
            self.stats_host.copy_(self.stats, non_blocking=True)
        self.stream.synchronize()
        pairs = int(self.stats_host[0])
        self.pair_ws = self._grow(self.pair_ws, max(1, lib.dgmr_splat_pair_workspace_size(n, pairs)))
        N.check(lib.dgmr_splat_render(scene, camera, N.ptr(framebuffer), N.ptr(self.frame_ws), self.frame_ws.numel(),
                                      N.ptr(self.pair_ws), self.pair_ws.numel(), pairs, N.ptr(self.stats), s),
                "splat render")
        self._last = (scene, camera, n, W, H, pairs)
        return pairs

    def frame(self) -> SplatFrame:
        """The last rendered frame, for splat_backward; valid until the next
        forward of this context."""
        scene, camera, n, W, H, pairs = self._last
        return SplatFrame(self.frame_ws, self.pair_ws, pairs, self.stats, scene, camera, n, W, H)
