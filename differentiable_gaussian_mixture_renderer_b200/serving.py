"""Serving the splat renderer: resident scenes, requests in flight on several
CUDA streams, no host synchronisation per request.

A request is (scene, camera).  Each of ``n_slots`` slots owns a stream, a
frame workspace, a pair workspace, a device framebuffer and a pinned host
image; a new request takes the least recently used slot once its previous
request has finished, so up to ``n_slots`` frames overlap on the GPU
(preprocess and sort of one with the blend of another, device-to-host copies
with compute).  The pair capacity of each (scene, resolution) is learnt from
the frames rendered so far; a frame that overflowed its capacity is rendered
again with the exact count before its result is handed out, so every result
equals the plain per-call render.
"""
from __future__ import annotations

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

    @classmethod
    def from_numpy(cls, scene, device) -> "GaussianScene":
        t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float32).to(device)
        return cls(t(scene.sh), t(scene.weights).reshape(-1), t(scene.centroids), t(scene.scales), t(scene.rotations),
                   int(scene.sh_degree))

    @property
    def n(self) -> int:
        return int(self.centroids.shape[0])

    def c_scene(self) -> N.Scene:
        return N.make_scene(self.shs, self.weights, self.centroids, self.scales, self.rotations, self.sh_degree)

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
    fb: torch.Tensor | None = None
    host: torch.Tensor | None = None
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
        if slot.fb is None or tuple(slot.fb.shape) != (3, H, W):
            slot.fb = torch.empty((3, H, W), dtype=torch.float32, device=dev)
            slot.host = None
        if to_host and slot.host is None:
            slot.host = torch.empty((3, H, W), dtype=torch.float32, pin_memory=True)
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
        N.check(self.lib.dgmr_splat_forward(scene.c_scene(), camera_struct(cam, req.background), N.ptr(slot.fb),
                                            N.ptr(slot.frame_ws), slot.frame_ws.numel(), N.ptr(slot.pair_ws),
                                            slot.pair_ws.numel(), cap, N.ptr(slot.stats), s.cuda_stream),
                "splat forward")
        slot.stats_host.copy_(slot.stats, non_blocking=True)
        if req.to_host:
            slot.host.copy_(slot.fb, non_blocking=True)

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
        req.image = slot.host if req.to_host else slot.fb
        req.meta["n_pairs"] = n_pairs
        self.completed.append(req)
        slot.request = None

    def drain(self):
        for slot in self.slots:
            if slot.request is not None:
                self._finish(slot)

    def start_clock(self):
        """Anchor device completion times to the host clock (streams idle)."""
        torch.cuda.synchronize(self.device)
        self.ref_event = torch.cuda.Event(enable_timing=True)
        self.ref_event.record(self.slots[0].stream)
        self.t0 = time.perf_counter()
        self.ref_event.synchronize()
