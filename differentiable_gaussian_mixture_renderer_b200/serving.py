"""Serving the splat renderer: resident scenes, requests in flight on several
CUDA streams, no host synchronisation per request.

A request is (scene, camera).  Each of ``n_slots`` slots owns a stream, a
frame workspace and a pair workspace; a new request takes the least recently
used slot once its previous request has finished, so up to ``n_slots`` frames
overlap on the GPU (preprocess and sort of one with the blend of another,
device-to-host copies with compute).  The pair capacity of each (scene,
resolution) is learnt from the frames rendered so far; a frame that
overflowed its capacity is rendered again with the exact count before its
result is handed out, so every result equals the plain per-call render.

Every request owns its result: its framebuffer (and pinned host image) are
leased from a pool of the server's and stay the request's until the caller
hands them back with ``Request.release()``; a result the caller keeps is never
written by a later request.  A caller that releases each result once it has
read it lets the server run on a fixed set of buffers.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _native as N


@dataclass
class GaussianScene:
    """Device-resident Gaussian mixture (float32, reference layouts)."""
    shs: torch.Tensor
    weights: torch.Tensor
    centroids: torch.Tensor
    scales: torch.Tensor
    rotations: torch.Tensor
    sh_degree: int
    formulation: str | None = None  # None = the splat renderer's Ots

    @classmethod
    def from_numpy(cls, scene, device) -> "GaussianScene":
        t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float32).to(device)
        return cls(t(scene.sh), t(scene.weights).reshape(-1), t(scene.centroids), t(scene.scales), t(scene.rotations),
                   int(scene.sh_degree), getattr(scene, "formulation", None))

    @property
    def n(self) -> int:
        return int(self.centroids.shape[0])

    def c_scene(self) -> N.Scene:
        return N.make_scene(self.shs, self.weights, self.centroids, self.scales, self.rotations, self.sh_degree,
                            self.formulation)

    def nbytes(self) -> int:
        return sum(t.numel() * t.element_size() for t in (self.shs, self.weights, self.centroids, self.scales,
                                                            self.rotations))


def camera_struct(cam, background=(0.0, 0.0, 0.0)) -> N.Camera:
    """dgmr_camera from a scene.Camera (numpy, torch layout)."""
    return N.make_camera(cam.view.reshape(-1), cam.proj.reshape(-1), cam.campos, background, cam.width, cam.height,
                         cam.tan_fovx, cam.tan_fovy)


@dataclass
class _Slot:
    stream: torch.cuda.Stream
    frame_ws: torch.Tensor | None = None
    pair_ws: torch.Tensor | None = None
    cap: int = 0
    stats: torch.Tensor | None = None
    stats_host: torch.Tensor | None = None
    done: torch.cuda.Event | None = None
    request: "Request | None" = None
    key: tuple = ()


@dataclass
class Request:
    scene_id: str
    camera: object
    background: tuple = (0.0, 0.0, 0.0)
    to_host: bool = True
    t_submit: float = 0.0
    t_done: float = 0.0
    image: torch.Tensor | None = None
    rerendered: bool = False
    slot: int = -1
    meta: dict = field(default_factory=dict)
    _release: object = None  # set by the server that leased the result buffers

    def release(self) -> None:
        """Hands the result buffers back to the server that rendered them; the
        request's ``image`` is gone afterwards.  Without this call the request
        simply keeps them."""
        if self._release is not None:
            self._release(self)
            self._release = None
        self.image = None


class RenderServer:
    def __init__(self, scenes: dict, device=None, n_slots: int = 3, capacity_margin: float = 1.25):
        self.device = torch.device(device or "cuda")
        self.scenes = scenes
        self.lib = N.lib()
        self.slots = [_Slot(torch.cuda.Stream(device=self.device)) for _ in range(n_slots)]
        self.next_slot = 0
        self.capacity: dict = {}
        self.margin = capacity_margin
        self.rerenders = 0
        self.completed: list[Request] = []
        self.ref_event = None
        self.t0 = 0.0
        self._pool: dict = {}  # (pinned, H, W) -> result buffers no request holds

    # ------------------------------------------------------------ result buffers
    def _lease(self, pinned: bool, H: int, W: int) -> torch.Tensor:
        free = self._pool.get((pinned, H, W))
        if free:
            return free.pop()
        if pinned:
            return torch.empty((3, H, W), dtype=torch.float32, pin_memory=True)
        return torch.empty((3, H, W), dtype=torch.float32, device=self.device)

    def _give_back(self, buf: torch.Tensor | None, pinned: bool) -> None:
        if buf is not None:
            self._pool.setdefault((pinned, int(buf.shape[1]), int(buf.shape[2])), []).append(buf)

    def _release_request(self, req: Request) -> None:
        self._give_back(req.meta.pop("_fb", None), False)
        self._give_back(req.meta.pop("_host", None), True)

    # ------------------------------------------------------------ buffers
    def _ensure(self, slot: _Slot, scene: GaussianScene, W: int, H: int, cap: int, to_host: bool):
        dev = self.device
        lib = self.lib
        fbytes = lib.dgmr_splat_frame_workspace_size(scene.n, W, H)
        if slot.frame_ws is None or slot.frame_ws.numel() < fbytes:
            slot.frame_ws = torch.empty(fbytes, dtype=torch.uint8, device=dev)
        pbytes = max(1, lib.dgmr_splat_pair_workspace_size(scene.n, cap))
        if slot.pair_ws is None or slot.pair_ws.numel() < pbytes:
            slot.pair_ws = torch.empty(pbytes, dtype=torch.uint8, device=dev)
        if slot.stats is None:
            slot.stats = torch.zeros(4, dtype=torch.int32, device=dev)
            slot.stats_host = torch.zeros(4, dtype=torch.int32, pin_memory=True)
        slot.cap = cap

    def estimate_capacity(self, scene_id: str, cam, slot_index: int | None = None) -> int:
        """Pair count of one frame (synchronous); seeds the capacity table.
        Runs on a free slot (``slot_index``, or after draining all slots)."""
        scene = self.scenes[scene_id]
        W, H = cam.width, cam.height
        if slot_index is None:
            self.drain()
            slot_index = 0
        slot = self.slots[slot_index]
        self._ensure(slot, scene, W, H, 0, False)
        with torch.cuda.stream(slot.stream):
            N.check(self.lib.dgmr_splat_preprocess(scene.c_scene(), camera_struct(cam), N.ptr(slot.frame_ws),
                                                   slot.frame_ws.numel(), N.ptr(slot.stats), slot.stream.cuda_stream),
                    "splat preprocess")
            slot.stats_host.copy_(slot.stats, non_blocking=True)
        slot.stream.synchronize()
        p = int(slot.stats_host[0])
        key = (scene_id, W, H)
        self.capacity[key] = max(self.capacity.get(key, 0), int(math.ceil(p * self.margin)) + 1024)
        return p

    # ------------------------------------------------------------ requests
    def _launch(self, slot: _Slot, req: Request, cap: int):
        scene = self.scenes[req.scene_id]
        cam = req.camera
        self._ensure(slot, scene, cam.width, cam.height, cap, req.to_host)
        s = slot.stream
        # the request's own result buffers (kept on a re-render)
        if "_fb" not in req.meta:
            req.meta["_fb"] = self._lease(False, cam.height, cam.width)
            if req.to_host:
                req.meta["_host"] = self._lease(True, cam.height, cam.width)
            req._release = self._release_request
        fb = req.meta["_fb"]
        N.check(self.lib.dgmr_splat_forward(scene.c_scene(), camera_struct(cam, req.background), N.ptr(fb),
                                            N.ptr(slot.frame_ws), slot.frame_ws.numel(), N.ptr(slot.pair_ws),
                                            slot.pair_ws.numel(), cap, N.ptr(slot.stats), s.cuda_stream),
                "splat forward")
        slot.stats_host.copy_(slot.stats, non_blocking=True)
        if req.to_host:
            req.meta["_host"].copy_(fb, non_blocking=True)

    def submit(self, req: Request) -> Request:
        idx = self.next_slot
        self.next_slot = (idx + 1) % len(self.slots)
        slot = self.slots[idx]
        if slot.request is not None:
            self._finish(slot)
        req.slot = idx
        req.t_submit = time.perf_counter()
        key = (req.scene_id, req.camera.width, req.camera.height)
        if key not in self.capacity:
            self.estimate_capacity(req.scene_id, req.camera, idx)
        with torch.cuda.stream(slot.stream):
            self._launch(slot, req, self.capacity[key])
            slot.done = torch.cuda.Event(enable_timing=True)
            slot.done.record(slot.stream)
        slot.request = req
        slot.key = key
        return req

    def _finish(self, slot: _Slot):
        req = slot.request
        slot.done.synchronize()
        n_pairs, flags = int(slot.stats_host[0]), int(slot.stats_host[1])
        if flags & N.FLAG_PAIR_OVERFLOW:
            # the frame needed more pairs than the capacity: render it again, exactly sized
            self.rerenders += 1
            req.rerendered = True
            self.capacity[slot.key] = max(self.capacity[slot.key], int(math.ceil(n_pairs * self.margin)) + 1024)
            with torch.cuda.stream(slot.stream):
                self._launch(slot, req, self.capacity[slot.key])
                slot.done = torch.cuda.Event(enable_timing=True)
                slot.done.record(slot.stream)
            slot.done.synchronize()
        if self.ref_event is not None:
            req.t_done = self.t0 + self.ref_event.elapsed_time(slot.done) * 1e-3
        else:
            req.t_done = time.perf_counter()
        if req.to_host:
            # the copy to the host has finished: the device framebuffer is free again
            self._give_back(req.meta.pop("_fb"), False)
            req.image = req.meta["_host"]
        else:
            req.image = req.meta["_fb"]
        req.meta["n_pairs"] = n_pairs
        self.completed.append(req)
        slot.request = None

    def drain(self):
        for slot in self.slots:
            if slot.request is not None:
                self._finish(slot)

    def release_buffers(self):
        """Finishes what is in flight and drops the slots' workspaces and the
        pooled result buffers (results still held by requests stay theirs)."""
        self.drain()
        self._pool.clear()
        for slot in self.slots:
            slot.frame_ws = slot.pair_ws = None

    def start_clock(self):
        """Anchor device completion times to the host clock (streams idle)."""
        torch.cuda.synchronize(self.device)
        self.ref_event = torch.cuda.Event(enable_timing=True)
        self.ref_event.record(self.slots[0].stream)
        self.t0 = time.perf_counter()
        self.ref_event.synchronize()


# ---------------------------------------------------------------------------
# Continuous batching over several resident scenes.
#
# Requests (render, or render + gradient against a caller-given image
# gradient) arrive at any time.  Whenever a slot (a CUDA stream with its own
# workspaces) is free, the queue head is cut into one batch -- as many waiting
# requests as fit the view/scene limits of one batched launch and the free
# HBM budget -- and launched with dgmr_splat_batch_forward (+ _backward).
# Requests that arrive while batches are on the GPU wait only for the next
# free slot; several batches run concurrently on their streams.  Every
# request owns its output buffers (image, gradients), written in place by the
# batched kernels, so a result is the same bits alone or in any mix: images
# bit-identical, gradients equal up to the order of the per-pixel atomics.
# A gradient request gets its own entry in the batch's scene table (same
# tensors, its own gradient outputs), so its gradients never mix with another
# request's.


class HbmBudget:
    """Bytes of device memory the server may hold for in-flight work.  A batch
    is admitted only if its reservation fits next to what is in flight."""

    def __init__(self, budget_bytes: int):
        self.budget = int(budget_bytes)
        self.in_use = 0
        self.peak = 0

    def fits(self, nbytes: int) -> bool:
        return self.in_use + int(nbytes) <= self.budget

    def reserve(self, nbytes: int) -> None:
        if not self.fits(nbytes):
            raise RuntimeError("reservation exceeds the HBM budget")
        self.in_use += int(nbytes)
        self.peak = max(self.peak, self.in_use)

    def release(self, nbytes: int) -> None:
        self.in_use = max(0, self.in_use - int(nbytes))


def form_batch(queue: list, max_views: int, max_scene_entries: int, cost, budget: HbmBudget):
    """Takes requests from the head of ``queue`` (arrival order, no
    reordering) while the batch stays within the view and scene-entry limits
    and ``cost(batch)`` (bytes) fits the budget.  Render requests of one scene
    share a scene entry; each gradient request has its own.  Returns
    (batch, bytes); the batch is empty when even the head does not fit."""
    batch, scenes = [], set()
    entries = 0
    nbytes = 0
    for req in queue:
        if len(batch) >= max_views:
            break
        new_entry = req.backward or req.scene_id not in scenes
        if new_entry and entries + 1 > max_scene_entries:
            break
        trial = batch + [req]
        c = cost(trial)
        if not budget.fits(c):
            break
        batch = trial
        nbytes = c
        if new_entry:
            entries += 1
        if not req.backward:
            scenes.add(req.scene_id)
    del queue[:len(batch)]
    return batch, nbytes


@dataclass
class ServeRequest:
    scene_id: str
    camera: object
    backward: bool = False
    grad_image: torch.Tensor | None = None  # [3,H,W] device, for gradient requests
    arrival: float = 0.0
    t_launch: float = 0.0
    t_done: float = 0.0
    image: torch.Tensor | None = None
    grads: tuple | None = None  # (sh, weights, centroids, scales, rotations)
    batch_size: int = 0
    rerendered: bool = False
    kind: str = "splat"  # "splat", or "march" (vol_marcher; NativeServer only)
    host_image: torch.Tensor | None = None  # optional pinned [3,H,W]: NativeServer copies the image there too
    status: int = 0


@dataclass
class _BatchSlot:
    stream: torch.cuda.Stream
    frame_ws: torch.Tensor | None = None
    pair_ws: torch.Tensor | None = None
    stats: torch.Tensor | None = None
    stats_host: torch.Tensor | None = None
    done: torch.cuda.Event | None = None
    batch: list = field(default_factory=list)
    tables: tuple = ()
    capacity: int = 0
    reserved: int = 0
    start: torch.cuda.Event | None = None


class ContinuousServer:
    """Continuous batching of render and gradient requests over resident scenes."""

    def __init__(self, scenes: dict, device=None, n_slots: int = 4, max_batch: int = 8,
                 hbm_budget_bytes: int | None = None, capacity_margin: float = 2.0):
        self.device = torch.device(device or "cuda")
        self.scenes = scenes
        self.lib = N.lib()
        self.slots = [_BatchSlot(torch.cuda.Stream(device=self.device)) for _ in range(n_slots)]
        self.max_batch = min(max_batch, N.BATCH_MAX_VIEWS)
        self.margin = capacity_margin
        if hbm_budget_bytes is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            hbm_budget_bytes = int(free * 0.8)
        self.budget = HbmBudget(hbm_budget_bytes)
        self.queue: list = []
        self.completed: list = []
        self.capacity: dict = {}  # (scene_id, W, H) -> pairs
        self._unit_cost: dict = {}  # (scene_id, W, H, backward) -> bytes of a one-request batch
        self.rerenders = 0
        self.batches = 0
        self.deferred = 0  # times the queue head waited for memory held by batches in flight
        self.reallocs = 0  # workspace growths (each one a fresh device allocation)
        self.log: list = []  # per completed batch: (requests, capacity, pairs, host seconds in flight)

    # ------------------------------------------------------------ sizing
    def _pairs(self, req) -> int:
        key = (req.scene_id, req.camera.width, req.camera.height)
        if key not in self.capacity:
            scene = self.scenes[req.scene_id]
            ws = torch.empty(max(1, self.lib.dgmr_splat_frame_workspace_size(scene.n, key[1], key[2])),
                             dtype=torch.uint8, device=self.device)
            stats = torch.zeros(4, dtype=torch.int32, device=self.device)
            N.check(self.lib.dgmr_splat_preprocess(scene.c_scene(), camera_struct(req.camera), N.ptr(ws), ws.numel(),
                                                   N.ptr(stats), N.stream_handle()), "splat preprocess")
            self.capacity[key] = int(math.ceil(int(stats[0].item()) * self.margin)) + 1024
        return self.capacity[key]

    def _tables(self, batch):
        entries, scene_of_entry, index = [], [], {}
        views = (N.BatchView * len(batch))()
        for k, req in enumerate(batch):
            if req.backward or req.scene_id not in index:
                if not req.backward:
                    index[req.scene_id] = len(entries)
                entries.append(self.scenes[req.scene_id].c_scene())
                scene_of_entry.append(req)
                e = len(entries) - 1
            else:
                e = index[req.scene_id]
            views[k].scene = e
            views[k].camera = camera_struct(req.camera)
        scenes = (N.Scene * len(entries))(*entries)
        return scenes, views, scene_of_entry

    def _exact_cost(self, batch) -> int:
        scenes, views, _ = self._tables(batch)
        cap = sum(self._pairs(r) for r in batch)
        fb, pb = C.c_size_t(0), C.c_size_t(0)
        N.check(self.lib.dgmr_splat_batch_workspace_size(scenes, len(scenes), views, len(views), cap, C.byref(fb),
                                                         C.byref(pb)), "batch workspace size")
        out = sum(12 * r.camera.width * r.camera.height for r in batch)
        grads = sum(self.scenes[r.scene_id].nbytes() for r in batch if r.backward)
        return int(fb.value) + int(pb.value) + out + grads

    def _cost(self, batch) -> int:
        """HBM a batch holds: the sum of its requests' one-request costs (every
        workspace part is linear in the views' slots, tiles, pixels and pairs;
        the per-request sum over-counts only the alignment padding)."""
        total = 0
        for r in batch:
            key = (r.scene_id, r.camera.width, r.camera.height, r.backward)
            c = self._unit_cost.get(key)
            if c is None:
                c = self._exact_cost([r])
                self._unit_cost[key] = c
            total += c
        return total

    # ------------------------------------------------------------ running
    def submit(self, req: ServeRequest) -> ServeRequest:
        if req.backward and (req.grad_image is None
                             or tuple(req.grad_image.shape) != (3, req.camera.height, req.camera.width)):
            raise ValueError("a gradient request needs grad_image [3, H, W]")
        self.queue.append(req)
        return req

    def _launch(self, slot: _BatchSlot, batch: list, capacity: int):
        scenes, views, owners = self._tables(batch)
        dev = self.device
        for k, req in enumerate(batch):
            if req.image is None:
                req.image = torch.empty((3, req.camera.height, req.camera.width), dtype=torch.float32, device=dev)
            views[k].framebuffer = req.image.data_ptr()
            if req.backward:
                views[k].grad_framebuffer = req.grad_image.data_ptr()
        grads = (N.SceneGrads * len(owners))()
        any_bwd = False
        for e, req in enumerate(owners):
            if req.backward:
                any_bwd = True
                sc = self.scenes[req.scene_id]
                if req.grads is None:
                    req.grads = (torch.empty_like(sc.shs), torch.empty_like(sc.weights), torch.empty_like(sc.centroids),
                                 torch.empty_like(sc.scales), torch.empty_like(sc.rotations))
                g = req.grads
                grads[e].sh, grads[e].weights, grads[e].centroids = g[0].data_ptr(), g[1].data_ptr(), g[2].data_ptr()
                grads[e].scales, grads[e].rotations = g[3].data_ptr(), g[4].data_ptr()
        fb, pb = C.c_size_t(0), C.c_size_t(0)
        N.check(self.lib.dgmr_splat_batch_workspace_size(scenes, len(scenes), views, len(views), capacity, C.byref(fb),
                                                         C.byref(pb)), "batch workspace size")
        if slot.frame_ws is None or slot.frame_ws.numel() < fb.value:
            slot.frame_ws = None
            slot.frame_ws = torch.empty(max(1, int(fb.value * 1.25)), dtype=torch.uint8, device=dev)
            self.reallocs += 1
        if slot.pair_ws is None or slot.pair_ws.numel() < pb.value:
            slot.pair_ws = None
            slot.pair_ws = torch.empty(max(1, int(pb.value * 1.25)), dtype=torch.uint8, device=dev)
            self.reallocs += 1
        if slot.stats is None:
            slot.stats = torch.zeros(4, dtype=torch.int32, device=dev)
            slot.stats_host = torch.zeros(4, dtype=torch.int32, pin_memory=True)
        s = slot.stream
        with torch.cuda.stream(s):
            slot.start = torch.cuda.Event(enable_timing=True)
            slot.start.record(s)
            N.check(self.lib.dgmr_splat_batch_forward(scenes, len(scenes), views, len(views), N.ptr(slot.frame_ws),
                                                      slot.frame_ws.numel(), N.ptr(slot.pair_ws), slot.pair_ws.numel(),
                                                      capacity, N.ptr(slot.stats), s.cuda_stream), "batch forward")
            slot.stats_host.copy_(slot.stats, non_blocking=True)
            if any_bwd:
                # render-only views and their scene entries carry null gradient pointers: skipped
                N.check(self.lib.dgmr_splat_batch_backward(scenes, len(scenes), views, len(views), grads,
                                                           N.ptr(slot.frame_ws), slot.frame_ws.numel(),
                                                           N.ptr(slot.pair_ws), slot.pair_ws.numel(), capacity,
                                                           s.cuda_stream), "batch backward")
            slot.done = torch.cuda.Event(enable_timing=True)
            slot.done.record(s)
        slot.batch = batch
        slot.tables = (scenes, views, grads)
        slot.capacity = capacity

    def _complete(self, slot: _BatchSlot, now: float):
        n_pairs, flags = int(slot.stats_host[0]), int(slot.stats_host[1])
        if flags & N.FLAG_PAIR_OVERFLOW:
            # more pairs than the learnt capacities: grow them and render the batch again with the
            # exact count, asynchronously -- the slot stays busy and completes on a later poll
            self.rerenders += 1
            grow = n_pairs / max(slot.capacity, 1)
            grown = set()  # each key grows once, however many of its requests the batch holds
            for req in slot.batch:
                req.rerendered = True
                key = (req.scene_id, req.camera.width, req.camera.height)
                if key in grown:
                    continue
                grown.add(key)
                self.capacity[key] = min(int(math.ceil(self.capacity[key] * max(self.margin, grow))), 0x7fffffff)
                self._unit_cost.pop((*key, False), None)
                self._unit_cost.pop((*key, True), None)
            self._launch(slot, slot.batch, n_pairs + 1024)
            return
        self.log.append((len(slot.batch), slot.capacity, n_pairs, now - slot.batch[0].t_launch,
                         slot.start.elapsed_time(slot.done), any(r.backward for r in slot.batch),
                         slot.batch[0].rerendered))
        for req in slot.batch:
            req.t_done = now
            req.batch_size = len(slot.batch)
            self.completed.append(req)
        self.budget.release(slot.reserved)
        slot.batch, slot.tables, slot.reserved = [], (), 0

    def poll(self) -> int:
        """Completes finished batches and launches new ones on free slots.
        Returns the number of requests in flight."""
        now = time.perf_counter()
        for slot in self.slots:
            if slot.batch and slot.done.query():
                self._complete(slot, now)
        for slot in self.slots:
            if slot.batch or not self.queue:
                continue
            batch, nbytes = form_batch(self.queue, self.max_batch, N.BATCH_MAX_SCENES, self._cost, self.budget)
            if not batch:
                if not any(s.batch for s in self.slots):
                    raise RuntimeError("a single request does not fit the HBM budget")
                self.deferred += 1
                break
            self.budget.reserve(nbytes)
            slot.reserved = nbytes
            t = time.perf_counter()
            for req in batch:
                req.t_launch = t
            self._launch(slot, batch, sum(self._pairs(r) for r in batch))
            self.batches += 1
        return sum(len(s.batch) for s in self.slots)

    def drain(self):
        while self.queue or any(s.batch for s in self.slots):
            if not self.poll():
                continue
            for slot in self.slots:
                if slot.batch:
                    slot.done.synchronize()
                    break


# ---------------------------------------------------------------------------
# The same server in native code: the queue, the batch cutting, the HBM
# admission, the capacity learning and the re-render of overflowed batches run
# in C++ behind dgmr_server_* (csrc/dgmr_server.cpp); Python only hands it
# device pointers and reads completions.  It also serves vol_marcher requests
# (kind="march"), forward and backward, batched with other marcher requests
# (a batch holds one kind).


class NativeServer:
    """Continuous batching of splat and vol_marcher requests by the library's
    C++ server.  Requests are ServeRequest objects as for ContinuousServer;
    each owns its outputs (image, gradients, optional pinned host copy), and a
    completed request's results equal the plain call's."""

    def __init__(self, scenes: dict, device=None, n_slots: int = 4, max_batch: int = 8,
                 hbm_budget_bytes: int | None = None, capacity_margin: float = 2.0, max_batch_pixels: int = 0):
        self.device = torch.device(device or "cuda")
        self.lib = N.lib()
        cfg = N.ServerConfig(self.device.index if self.device.index is not None else torch.cuda.current_device(),
                             n_slots, max_batch, 0, int(hbm_budget_bytes or 0), capacity_margin, int(max_batch_pixels))
        handle = C.c_void_p()
        N.check(self.lib.dgmr_server_create(C.byref(cfg), C.byref(handle)), "server create")
        self._h = handle
        # completions carry the server's clock: align it with this process's perf_counter
        self._t0 = time.perf_counter() - self.lib.dgmr_server_now(self._h)
        self.scenes = scenes
        self._index = {}
        self._c_scenes = {}
        for sid, sc in scenes.items():
            self._c_scenes[sid] = sc.c_scene()
            idx = C.c_int32()
            N.check(self.lib.dgmr_server_add_scene(self._h, C.byref(self._c_scenes[sid]), C.byref(idx)), "server scene")
            self._index[sid] = idx.value
        self._inflight: dict = {}
        self._next_tag = 1
        self._buf = (N.ServerCompletion * 64)()
        self.completed: list = []

    def submit(self, req: ServeRequest) -> ServeRequest:
        sc = self.scenes[req.scene_id]
        H, W = req.camera.height, req.camera.width
        if req.kind not in ("splat", "march"):
            raise ValueError("kind must be 'splat' or 'march'")
        if req.backward and (req.grad_image is None or tuple(req.grad_image.shape) != (3, H, W)
                             or req.grad_image.dtype != torch.float32 or not req.grad_image.is_contiguous()):
            raise ValueError("a gradient request needs a contiguous float32 grad_image [3, H, W]")
        if req.image is None:
            req.image = torch.empty((3, H, W), dtype=torch.float32, device=self.device)
        if req.backward and req.grads is None:
            req.grads = (torch.empty_like(sc.shs), torch.empty_like(sc.weights), torch.empty_like(sc.centroids),
                         torch.empty_like(sc.scales), torch.empty_like(sc.rotations))
        r = N.ServerRequest()
        r.kind = N.SERVE_MARCH if req.kind == "march" else N.SERVE_SPLAT
        r.scene = self._index[req.scene_id]
        r.camera = camera_struct(req.camera)
        r.framebuffer = req.image.data_ptr()
        if req.backward:
            r.grad_image = req.grad_image.data_ptr()
            g = req.grads
            r.grads = N.SceneGrads(g[0].data_ptr(), g[1].data_ptr(), g[2].data_ptr(), g[3].data_ptr(), g[4].data_ptr())
        if req.host_image is not None:
            if not req.host_image.is_pinned() or tuple(req.host_image.shape) != (3, H, W):
                raise ValueError("host_image must be pinned float32 [3, H, W]")
            r.host_image = req.host_image.data_ptr()
        r.tag = self._next_tag
        self._next_tag += 1
        # work queued on torch's stream that produced the inputs must be done before the server's streams read them
        torch.cuda.current_stream(self.device).synchronize()
        N.check(self.lib.dgmr_server_submit(self._h, C.byref(r)), "server submit")
        self._inflight[r.tag] = req
        return req

    def _collect(self, n: int) -> None:
        failed = None
        for k in range(n):
            c = self._buf[k]
            req = self._inflight.pop(c.tag)
            req.t_launch = self._t0 + c.launch_s
            req.t_done = self._t0 + c.done_s
            req.batch_size = c.batch_size
            req.rerendered = bool(c.rerendered)
            req.status = c.status
            self.completed.append(req)
            if c.status != N.DGMR_OK and failed is None:
                failed = c.status
        if failed is not None:
            N.check(failed, "served request")

    def poll(self) -> int:
        """Completes finished batches, launches new ones; returns the number of
        requests still queued or in flight."""
        self._collect(self.lib.dgmr_server_poll(self._h, self._buf, len(self._buf)))
        return len(self._inflight)

    def drain(self) -> None:
        while self._inflight:
            self._collect(self.lib.dgmr_server_wait(self._h, self._buf, len(self._buf)))

    def stats(self) -> dict:
        st = N.ServerStats()
        N.check(self.lib.dgmr_server_get_stats(self._h, C.byref(st)), "server stats")
        return {f: getattr(st, f) for f, _ in N.ServerStats._fields_ if f != "reserved"}

    def close(self) -> None:
        if self._h:
            self.drain()
            self.lib.dgmr_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            if getattr(self, "_h", None):
                self.lib.dgmr_server_destroy(self._h)
                self._h = None
        except Exception:
            pass
