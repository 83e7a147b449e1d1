"""Batched multi-view rendering: many cameras of several resident scenes,
uneven Gaussian counts and resolutions, in one launch sequence, optionally
captured in a CUDA graph, with an autotuner over the batch depth and, for
the splat renderer, the blend's pixel-block size -- for the splat renderer
(``kind="splat"``) and the volume marcher (``kind="march"``).

The reference renders one view per call (splat_forward.cu:30-338; its
vol_marcher.apply, python_bindings/vol_marcher.py:19-65, marches one camera);
here a ``BatchPlan`` holds everything one batch needs (view table,
workspaces, framebuffers, gradient buffers), so a forward (and backward) of
the whole batch is two C calls -- ``dgmr_splat_batch_forward`` /
``_backward``, or ``dgmr_vm_batch_forward`` / ``_backward`` -- that allocate
nothing and never synchronise the host, which is what lets a plan be
captured once and replayed.  Every view's image is bit-identical to rendering
it alone; per-scene gradients are the sum over that scene's views.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field

import torch

from . import _native as N
from .serving import GaussianScene, camera_struct


@dataclass
class BatchPlan:
    scene_ids: list
    views: list  # (scene_id, camera)
    c_scenes: object
    c_views: object
    frame_ws: torch.Tensor
    pair_ws: torch.Tensor
    capacity: int
    stats: torch.Tensor
    framebuffers: list
    grad_framebuffers: list = field(default_factory=list)
    grads: dict = field(default_factory=dict)  # scene_id -> (g_sh, g_w, g_mu, g_s, g_q)
    c_grads: object = None
    graph: torch.cuda.CUDAGraph | None = None
    stream: torch.cuda.Stream | None = None

    @property
    def n_views(self) -> int:
        return len(self.views)

    def overflowed(self) -> bool:
        """Device flag of the last run (synchronises)."""
        return bool(int(self.stats[1].item()) & N.FLAG_PAIR_OVERFLOW)

    def n_pairs(self) -> int:
        return int(self.stats[0].item())


class BatchRenderer:
    """Resident scenes rendered in batches of views, by the splat renderer
    (``kind="splat"``) or the volume marcher (``kind="march"``, float32,
    full render mode)."""

    # sides of the splat blend's pixel blocks (dgmr_batch_view.blend_block);
    # 0 leaves the choice to the library
    BLEND_BLOCKS = (8, 16)

    def __init__(self, scenes: dict, device=None, capacity_margin: float = 1.1, kind: str = "splat", blend_block: int = 0):
        if kind not in ("splat", "march"):
            raise ValueError("kind must be 'splat' or 'march'")
        if blend_block not in (0,) + self.BLEND_BLOCKS:
            raise ValueError(f"blend_block must be 0 or one of {self.BLEND_BLOCKS}")
        self.device = torch.device(device or "cuda")
        self.scenes: dict = scenes
        self.lib = N.lib()
        self.margin = capacity_margin
        self.kind = kind
        self.blend_block = blend_block
        pre = "dgmr_splat_batch_" if kind == "splat" else "dgmr_vm_batch_"
        self._c_size = getattr(self.lib, pre + "workspace_size")
        self._c_pre = getattr(self.lib, pre + "preprocess")
        self._c_fwd = getattr(self.lib, pre + "forward")
        self._c_bwd = getattr(self.lib, pre + "backward")

    # ------------------------------------------------------------ planning
    def _tables(self, views, backward: bool):
        scene_ids = []
        for sid, _ in views:
            if sid not in scene_ids:
                scene_ids.append(sid)
        if len(views) > N.BATCH_MAX_VIEWS or len(scene_ids) > N.BATCH_MAX_SCENES:
            raise ValueError(f"a batch holds at most {N.BATCH_MAX_VIEWS} views of {N.BATCH_MAX_SCENES} scenes")
        c_scenes = (N.Scene * len(scene_ids))(*[self.scenes[s].c_scene() for s in scene_ids])
        c_views = (N.BatchView * len(views))()
        for k, (sid, cam) in enumerate(views):
            c_views[k].scene = scene_ids.index(sid)
            c_views[k].blend_block = self.blend_block if self.kind == "splat" else 0
            c_views[k].camera = camera_struct(cam)
        return scene_ids, c_scenes, c_views

    def _sizes(self, c_scenes, c_views, cap: int):
        fb, pb = C.c_size_t(0), C.c_size_t(0)
        N.check(self._c_size(c_scenes, len(c_scenes), c_views, len(c_views), cap, C.byref(fb), C.byref(pb)),
                "batch workspace size")
        return int(fb.value), int(pb.value)

    def count_pairs(self, views) -> int:
        """Pairs of the whole batch (preprocess only; synchronises)."""
        scene_ids, c_scenes, c_views = self._tables(views, False)
        fbytes, _ = self._sizes(c_scenes, c_views, 0)
        ws = torch.empty(max(fbytes, 1), dtype=torch.uint8, device=self.device)
        stats = torch.zeros(4, dtype=torch.int32, device=self.device)
        N.check(self._c_pre(c_scenes, len(c_scenes), c_views, len(c_views), N.ptr(ws), fbytes, N.ptr(stats),
                            N.stream_handle()), "batch preprocess")
        return int(stats[0].item())

    def plan(self, views, backward: bool = False, capacity: int | None = None) -> BatchPlan:
        """Buffers for one batch.  ``views`` is a list of (scene_id, camera)."""
        scene_ids, c_scenes, c_views = self._tables(views, backward)
        if capacity is None:
            capacity = int(math.ceil(self.count_pairs(views) * self.margin)) + 4096
        fbytes, pbytes = self._sizes(c_scenes, c_views, capacity)
        dev = self.device
        frame_ws = torch.empty(max(fbytes, 1), dtype=torch.uint8, device=dev)
        pair_ws = torch.empty(max(pbytes, 1), dtype=torch.uint8, device=dev)
        fbs = [torch.empty((3, cam.height, cam.width), dtype=torch.float32, device=dev) for _, cam in views]
        for k, fb in enumerate(fbs):
            c_views[k].framebuffer = fb.data_ptr()
        p = BatchPlan(scene_ids, list(views), c_scenes, c_views, frame_ws, pair_ws, capacity,
                      torch.zeros(4, dtype=torch.int32, device=dev), fbs)
        if backward:
            p.grad_framebuffers = [torch.zeros_like(fb) for fb in fbs]
            for k, g in enumerate(p.grad_framebuffers):
                c_views[k].grad_framebuffer = g.data_ptr()
            p.c_grads = (N.SceneGrads * len(scene_ids))()
            for j, sid in enumerate(scene_ids):
                sc = self.scenes[sid]
                g = (torch.empty_like(sc.shs), torch.empty_like(sc.weights), torch.empty_like(sc.centroids),
                     torch.empty_like(sc.scales), torch.empty_like(sc.rotations))
                p.grads[sid] = g
                p.c_grads[j].sh, p.c_grads[j].weights, p.c_grads[j].centroids = (t.data_ptr() for t in g[:3])
                p.c_grads[j].scales, p.c_grads[j].rotations = g[3].data_ptr(), g[4].data_ptr()
        return p

    # ------------------------------------------------------------ running
    def forward(self, p: BatchPlan, stream: torch.cuda.Stream | None = None):
        s = N.stream_handle(stream)
        N.check(self._c_fwd(p.c_scenes, len(p.c_scenes), p.c_views, p.n_views, N.ptr(p.frame_ws), p.frame_ws.numel(),
                            N.ptr(p.pair_ws), p.pair_ws.numel(), p.capacity, N.ptr(p.stats), s), "batch forward")

    def backward(self, p: BatchPlan, stream: torch.cuda.Stream | None = None):
        if p.c_grads is None:
            raise ValueError("plan was made without backward buffers")
        s = N.stream_handle(stream)
        args = [p.c_scenes, len(p.c_scenes), p.c_views, p.n_views, p.c_grads, N.ptr(p.frame_ws), p.frame_ws.numel(),
                N.ptr(p.pair_ws), p.pair_ws.numel(), p.capacity]
        if self.kind == "march":
            args.append(N.ptr(p.stats))  # the step-limit flag
        N.check(self._c_bwd(*args, s), "batch backward")

    def capture(self, p: BatchPlan, backward: bool = False) -> BatchPlan:
        """Capture forward (+ backward) of the plan in a CUDA graph.  Replays
        read the plan's current inputs (scene tensors, grad framebuffers)."""
        p.stream = torch.cuda.Stream(device=self.device)
        p.stream.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(p.stream):  # one eager run first: sizes are right, nothing lazy inside capture
            self.forward(p, p.stream)
            if backward:
                self.backward(p, p.stream)
        p.stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=p.stream):
            self.forward(p, p.stream)
            if backward:
                self.backward(p, p.stream)
        p.graph = g
        return p

    def replay(self, p: BatchPlan):
        """Replays the captured graph on the plan's stream (ordered after the
        caller's current stream)."""
        if p.graph is None:
            raise ValueError("plan has no graph; call capture() first")
        p.stream.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(p.stream):
            p.graph.replay()
        torch.cuda.current_stream(self.device).wait_stream(p.stream)


def chunks(views, depth: int):
    """Consecutive groups of at most ``depth`` views (and 16 scenes)."""
    out, cur, scenes = [], [], set()
    for v in views:
        if len(cur) >= depth or (v[0] not in scenes and len(scenes) >= N.BATCH_MAX_SCENES):
            out.append(cur)
            cur, scenes = [], set()
        cur.append(v)
        scenes.add(v[0])
    if cur:
        out.append(cur)
    return out


def autotune(renderer: BatchRenderer, views, depths=(1, 4, 8, 16, 32, 48, 64), backward: bool = False, reps: int = 3,
             blend_blocks=None):
    """Picks the batch depth and (splat renderer) the blend block side for a
    view set of at most 64 views with the library's autotuner
    (``dgmr_batch_autotune``): each candidate renders the whole set, cut into
    consecutive batches of at most ``depth`` views, forward (and backward),
    timed with CUDA events on one stream.  Returns ((best_depth, best_block),
    {(depth, block): ms}) and leaves ``renderer.blend_block`` at the best side.
    ``blend_blocks`` defaults to BatchRenderer.BLEND_BLOCKS for the splat
    renderer and (0,) for the marcher.  Identical results for every setting;
    only the launch structure changes."""
    if blend_blocks is None:
        blend_blocks = BatchRenderer.BLEND_BLOCKS if renderer.kind == "splat" else (0,)
    depths = [d for d in depths if d <= N.BATCH_MAX_VIEWS]
    if not depths or not blend_blocks:
        raise ValueError("autotune needs at least one depth and one blend block")
    p = renderer.plan(views, backward=backward)
    d_arr = (C.c_int32 * len(depths))(*depths)
    b_arr = (C.c_int32 * len(blend_blocks))(*blend_blocks)
    ms = (C.c_float * (len(depths) * len(blend_blocks)))()
    best_d, best_b = C.c_int32(0), C.c_int32(0)
    kind = N.SERVE_SPLAT if renderer.kind == "splat" else N.SERVE_MARCH
    N.check(renderer.lib.dgmr_batch_autotune(kind, p.c_scenes, len(p.c_scenes), p.c_views, p.n_views,
                                             p.c_grads if backward else None, d_arr, len(depths), b_arr,
                                             len(blend_blocks), reps, N.ptr(p.frame_ws), p.frame_ws.numel(),
                                             N.ptr(p.pair_ws), p.pair_ws.numel(), p.capacity, ms, C.byref(best_d),
                                             C.byref(best_b), N.stream_handle()), "batch autotune")
    timings = {(d, b): float(ms[i * len(blend_blocks) + j]) for i, d in enumerate(depths)
               for j, b in enumerate(blend_blocks)}
    renderer.blend_block = int(best_b.value)
    del p
    return (int(best_d.value), int(best_b.value)), timings
