#!/usr/bin/env python
"""Served splat renders/s at 1080p with 1M Gaussians on B200.

Workload (one step = one batch of ``--batch`` render requests): a resident
scene of 1,000,000 Gaussians drawn as the reference's configuration 0
(centroids U[-1,1]^3, scales log-uniform [0.005, 0.05], random unit
quaternions, opacity sigmoid(N(0,1)), RGB as SH degree 0), requests are
random cameras on a sphere of radius 2.5-4 around it, 1920x1080, 60 degree
vertical field of view.  Synthetic seeded data (no dataset exists for this
path).

Legs:
  value     served renders/s, images left in HBM (RenderServer, several
            streams, no per-request host sync)
  e2e       the same through the public API with every image copied to
            pinned host memory inside the timed region
  plain     the plain per-call path: one request at a time, pair count read
            back per call (the reference's .item()), image copied to host
  roofline  the blend kernel re-run alone under CUDA events
  cpu       the CPU oracle (restated reference algorithm) on one frame

``--impl reference`` times the CPU restatement of the reference's path on all
host threads instead (the reference itself cannot be built here: its
git-fetched dependencies are absent).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "served renders/s + p50/p99 ms vs plain per-call splat, 1080p, 1M Gaussians"
UNIT = "renders/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--gaussians", type=int, default=1_000_000)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--batch", type=int, default=8, help="requests per step")
    ap.add_argument("--slots", type=int, default=4, help="requests in flight")
    ap.add_argument("--plain", type=int, default=64, help="plain per-call requests")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--python-server", action="store_true",
                    help="--workload serving: the Python ContinuousServer instead of the C++ server")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the short vol_marcher (100k, 512x512; 16 views of 64x64 batched), vol_raster, batched "
                         "(c3) and serving (c4) runs of the headline line")
    ap.add_argument("--workload", choices=["served", "batched", "marcher", "raster", "serving", "configs"], default="served",
                    help="served: the headline line (default); batched: 3 scenes x 16 views, mixed resolutions, "
                         "forward+backward under CUDA graphs; marcher: vol_marcher forward+backward, 100k, 512x512; "
                         "raster: vol_raster forward, 100k, 512x512; "
                         "serving: 8 scenes, Poisson 200 req/s, mixed resolutions, 20%% gradient requests; "
                         "configs: per-call GPU and oracle timings of the parity configurations")
    return ap.parse_args()


def workload(args):
    return {"workload": f"splat forward, {args.gaussians} Gaussians (config-0 distribution), {args.width}x{args.height}, "
                        f"random cameras r=2.5-4, {args.batch} requests/step",
            "n_gaussians": args.gaussians, "width": args.width, "height": args.height, "requests_per_step": args.batch,
            "slots_in_flight": args.slots,
            "l2": "working set > 126 MB L2 (~9M pairs x 32 B of binning buffers per frame)"}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        if not self.path or not os.path.exists(self.path):
            return out
        sms, maxs, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sms.append(float(parts[1]))
                maxs.append(float(parts[2]))
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        os.unlink(self.path)
        if sms:
            out = {"sm_mhz": statistics.median(sms), "sm_max_mhz": max(maxs), "reasons": sorted(reasons),
                   "samples": len(sms)}
        return out


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_value(name: str, key: str):
    """A per-launch figure ("key: value" line) from a committed ncu summary, if any."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(path):
            if line.startswith(key + ":"):
                return float(line.split(":", 1)[1].split()[0])
    except (OSError, ValueError):
        pass
    return None


SMS = 148  # B200


def issue_roof(warp_inst, ms, clocks):
    """Warp instructions issued per second against the issue roof: one warp
    instruction per cycle on each of the 4 schedulers of the 148 SMs, at the
    median SM clock sampled during the run (the maximum if none was read)."""
    if not warp_inst or not ms:
        return None
    mhz = (clocks or {}).get("sm_mhz") or (clocks or {}).get("sm_max_mhz") or 1965.0
    achieved = warp_inst / (ms * 1e-3)
    peak = SMS * 4 * mhz * 1e6
    return {"achieved": achieved, "peak": peak, "unit": "warp inst/s", "frac": achieved / peak,
            "warp_instructions_per_launch": warp_inst, "sm_mhz": mhz}


def cpu_baseline(args, cams):
    from oracle import oracle as O
    from differentiable_gaussian_mixture_renderer_b200 import scene as S
    sc = S.make_scene(args.gaussians, seed=0)
    O.splat_forward(sc, cams[0], want_keys=False)  # warm
    t = time.perf_counter()
    frames = 0
    for cam in cams[:2]:
        O.splat_forward(sc, cam, want_keys=False)
        frames += 1
        if time.perf_counter() - t > 20:
            break
    dt = time.perf_counter() - t
    return {"value": frames / dt, "unit": UNIT, "cores": O.num_threads(), "kind": "port",
            "sample": f"{frames} full frame(s) of the same workload (oracle splat forward, OpenMP)"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from differentiable_gaussian_mixture_renderer_b200 import scene as S
    from oracle import oracle as O
    sc = S.make_scene(args.gaussians, seed=0)
    cams = S.random_cameras(args.warmup + args.steps, args.width, args.height, seed=1)
    for cam in cams[:args.warmup]:
        O.splat_forward(sc, cam, want_keys=False)
    t = time.perf_counter()
    for cam in cams[args.warmup:]:
        O.splat_forward(sc, cam, want_keys=False)
    dt = time.perf_counter() - t
    value = args.steps / dt
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(workload(args), requests_per_step=1,
                           note="CPU restatement of the reference's splat path (oracle/, OpenMP); the reference "
                                "cannot be built here (its dependencies are fetched by git at build time)"),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": O.num_threads(), "kind": "port",
                             "sample": f"one full frame per step, {args.steps} steps"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def pct(xs, q):
    xs = sorted(xs)
    if not xs:
        return None
    k = (len(xs) - 1) * q / 100.0
    lo, hi = math.floor(k), math.ceil(k)
    return xs[lo] + (xs[hi] - xs[lo]) * (k - lo)


def replica_totals(ms_local: float, units_local: int, world: int, reduce_max, reduce_sum):
    """Whole-job numbers of N independent replicas: the slowest rank's device
    time and the units all ranks processed.  reduce_max / reduce_sum combine a
    float over the ranks (identity for one rank)."""
    ms = reduce_max(float(ms_local)) if world > 1 else float(ms_local)
    units = reduce_sum(float(units_local)) if world > 1 else float(units_local)
    return ms, units, units / (ms * 1e-3)


def run_ours(args):
    import torch
    import torch.distributed as dist
    from differentiable_gaussian_mixture_renderer_b200 import _native as N
    from differentiable_gaussian_mixture_renderer_b200 import scene as S
    from differentiable_gaussian_mixture_renderer_b200 import splat
    from differentiable_gaussian_mixture_renderer_b200 import serving
    from differentiable_gaussian_mixture_renderer_b200.serving import GaussianScene, RenderServer, Request

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def over_ranks(op):
        def reduce(x: float) -> float:
            t = torch.tensor([x], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=op)
            return float(t.item())
        return reduce

    max_over_ranks = over_ranks(dist.ReduceOp.MAX) if world > 1 else (lambda x: x)
    sum_over_ranks = over_ranks(dist.ReduceOp.SUM) if world > 1 else (lambda x: x)

    lib = N.lib()
    sc_np = S.make_scene(args.gaussians, seed=0)
    scene = GaussianScene.from_numpy(sc_np, dev)
    n_req = (args.warmup + args.steps) * args.batch
    cams = S.random_cameras(2 * n_req + args.plain + 4, args.width, args.height, seed=1 + 1000 * rank)
    server = RenderServer({"scene": scene}, dev, n_slots=args.slots)
    for cam in cams[:4]:
        server.estimate_capacity("scene", cam)

    # ---------------------------------------------------------------- value leg
    def release_done(upto: list):
        # each result is read (kept in HBM / pinned memory) and handed back, so the
        # server cycles through a fixed set of leased buffers
        while upto[0] < len(server.completed):
            server.completed[upto[0]].release()
            upto[0] += 1

    def served_leg(cam_list, to_host: bool):
        done = [0]
        for i in range(args.warmup * args.batch):
            server.submit(Request("scene", cam_list[i], to_host=to_host))
            release_done(done)
        server.drain()
        release_done(done)
        server.completed.clear()
        done = [0]
        barrier()
        launches0 = lib.dgmr_launch_count()
        start = torch.cuda.Event(enable_timing=True)
        end = torch.cuda.Event(enable_timing=True)
        server.start_clock()
        start.record(server.slots[0].stream)
        t_wall = time.perf_counter()
        for i in range(args.steps * args.batch):
            server.submit(Request("scene", cam_list[args.warmup * args.batch + i], to_host=to_host))
            release_done(done)
        server.drain()
        release_done(done)
        s0 = server.slots[0].stream
        for sl in server.slots[1:]:
            s0.wait_stream(sl.stream)
        end.record(s0)
        end.synchronize()
        wall = time.perf_counter() - t_wall
        barrier()
        ms = start.elapsed_time(end)
        lat = [(r.t_done - r.t_submit) * 1e3 for r in server.completed]
        return ms, wall, lat, lib.dgmr_launch_count() - launches0, sum(r.rerendered for r in server.completed)

    with ClockSampler(local) as clk:
        ms_value, wall_value, lat_value, launches, rerenders = served_leg(cams[:n_req], to_host=False)
        ms_e2e, wall_e2e, lat_e2e, _, _ = served_leg(cams[n_req:2 * n_req], to_host=True)
    local_renders = args.steps * args.batch
    ms_value, _, value = replica_totals(ms_value, local_renders, world, max_over_ranks, sum_over_ranks)
    ms_e2e, _, e2e_value = replica_totals(ms_e2e, local_renders, world, max_over_ranks, sum_over_ranks)

    # ---------------------------------------------------------------- the C++ server, same workload
    # (continuous batching: requests cut into batches of the batched entry points; host clock
    # from the first submission to the last completion, images to pinned host memory)
    native = None
    if not args.no_extras:
        # at this frame size views gain nothing from sharing a launch sequence: one view per batch,
        # args.slots batches in flight (smaller requests would still be batched)
        nserver = serving.NativeServer({"scene": scene}, dev, n_slots=args.slots, max_batch=args.batch,
                                       max_batch_pixels=args.width * args.height)
        hosts = [torch.empty((3, args.height, args.width), dtype=torch.float32, pin_memory=True)
                 for _ in range(2 * args.batch)]
        fbs = [torch.empty((3, args.height, args.width), dtype=torch.float32, device=dev) for _ in range(2 * args.batch)]

        def native_leg(cam_list, to_host):
            reqs = []
            for i, cam in enumerate(cam_list):
                r = serving.ServeRequest("scene", cam)
                r.image = fbs[i % len(fbs)]
                r.host_image = hosts[i % len(hosts)] if to_host else None
                reqs.append(r)
            for r in reqs[:2 * args.batch]:  # warm-up: capacities learnt, workspaces grown
                nserver.submit(r)
            nserver.drain()
            torch.cuda.synchronize(dev)
            t = time.perf_counter()
            for k, r in enumerate(reqs):
                # a result buffer is reused 2 x batch requests later: wait for its request first
                if k >= len(fbs):
                    while reqs[k - len(fbs)].t_done == 0.0:
                        nserver.poll()
                r.t_done = 0.0
                nserver.submit(r)
                nserver.poll()
            nserver.drain()
            torch.cuda.synchronize(dev)
            dt = time.perf_counter() - t
            lat = [(r.t_done - r.t_launch) * 1e3 for r in reqs]
            return len(reqs) / dt, lat, float(np.mean([r.batch_size for r in reqs]))

        nv, nlat, nbatch = native_leg(cams[:n_req], False)
        ne, nlat_e, nbatch_e = native_leg(cams[n_req:2 * n_req], True)
        st = nserver.stats()
        nserver.close()
        del nserver, hosts, fbs
        native = {"value": nv, "e2e": ne, "unit": UNIT, "mean_batch": nbatch, "launch_to_done_ms_p50": pct(nlat, 50),
                  "launch_to_done_ms_p99": pct(nlat, 99), "e2e_launch_to_done_ms_p50": pct(nlat_e, 50),
                  "rerenders": st["rerenders"],
                  "note": "the C++ continuous-batching server (dgmr_server_*, batches capped at one frame's pixels, "
                          "slots_in_flight batches in flight), host clock over the same number of requests; e2e with "
                          "each image copied to pinned host memory"}

    # ---------------------------------------------------------------- plain per-call leg
    # one request at a time on one stream, the reference's pattern: preprocess, the pair count
    # read back, binning + blend, the image copied to pinned host memory and waited for; the
    # workspaces grow once and are kept (no per-call allocation), as the C++ viewer interface does
    plain_cams = cams[2 * n_req:2 * n_req + args.plain]
    ctx = splat.SplatContext(dev)
    fb_plain = torch.empty((3, args.height, args.width), dtype=torch.float32, device=dev)
    host_plain = torch.empty((3, args.height, args.width), dtype=torch.float32, pin_memory=True)

    def plain_call(cam):
        ctx.forward(scene.shs, scene.weights, scene.centroids, scene.scales, scene.rotations,
                    serving.camera_struct(cam), fb_plain, scene.sh_degree)
        with torch.cuda.stream(ctx.stream):
            host_plain.copy_(fb_plain, non_blocking=True)
        ctx.stream.synchronize()

    for cam in cams[:max(args.warmup, 3)]:  # grows the workspaces to their steady size
        plain_call(cam)
    lat_plain = []
    barrier()
    for cam in plain_cams:
        t = time.perf_counter()
        plain_call(cam)
        lat_plain.append((time.perf_counter() - t) * 1e3)
    plain_rps = len(lat_plain) / (sum(lat_plain) * 1e-3) * world if lat_plain else None
    plain_rps_p50 = 1e3 / pct(lat_plain, 50) * world if lat_plain else None

    # ---------------------------------------------------------------- roofline of the blend
    cam = cams[0]
    fb, frame = splat.splat_forward(scene.shs, scene.weights, scene.centroids, scene.scales, scene.rotations, cam.view,
                                    cam.proj, cam.campos, (0.0, 0.0, 0.0), cam.width, cam.height, cam.tan_fovx,
                                    cam.tan_fovy, scene.sh_degree)
    torch.cuda.synchronize(dev)
    n_pairs = int(frame.stats[0].item())
    stream = torch.cuda.current_stream(dev)
    reps = 10
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)  # 2x the 126 MB L2
    for _ in range(2):
        N.check(lib.dgmr_splat_blend(frame.camera, frame.n, N.ptr(fb), *frame.ws_args(), frame.pair_capacity,
                                     stream.cuda_stream), "blend")
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(reps)]
    for e0, e1 in ev:  # each launch timed alone, L2 flushed before it
        flush.zero_()
        e0.record(stream)
        N.check(lib.dgmr_splat_blend(frame.camera, frame.n, N.ptr(fb), *frame.ws_args(), frame.pair_capacity,
                                     stream.cuda_stream), "blend")
        e1.record(stream)
    ev[-1][1].synchronize()
    blend_ms = sum(e0.elapsed_time(e1) for e0, e1 in ev) / reps
    del flush
    tiles = ((args.width + 15) // 16) * ((args.height + 15) // 16)
    px = args.width * args.height
    # algorithmic bytes of one blend launch: per pair its 32-byte record and 8-byte list entry,
    # per tile its range (8 B), per pixel its colour (12 B)
    blend_bytes = 40 * n_pairs + 8 * tiles + 12 * px
    # the same with everything the kernel touches: 4 B list id + 32 B record + 12 B rgb per pair,
    # and per pixel the final transmittance and contributor count the backward reads
    blend_bytes_touched = 48 * n_pairs + 8 * tiles + 20 * px
    peak, peak_kind = peaks()
    achieved = blend_bytes / (blend_ms * 1e-3) / 1e9
    # the committed ncu capture is of this frame at the default workload only
    default_workload = (args.gaussians, args.width, args.height) == (1_000_000, 1920, 1080)
    blend_profile = "splat_blend_1080p_1M.txt"
    traffic = profiled_value(blend_profile, "dram_bytes_per_launch") if default_workload else None
    warp_inst = profiled_value(blend_profile, "warp_instructions_per_launch") if default_workload else None

    # ---------------------------------------------------------------- the other workloads, short runs
    extras = {}
    if world == 1 and not args.no_extras:
        del fb, frame, ctx, fb_plain, host_plain
        server.release_buffers()
        extras["vol_marcher_c2"] = measure_marcher(dev, n_cams=3)
        extras["vol_marcher_batched_small_views"] = measure_marcher_batched(dev)
        extras["vol_raster_c2_scene"] = measure_vol_raster(dev, n_cams=3)
        extras["batched_c3"] = measure_batched(dev, steps=3, warmup=2)
        extras["serving_c4"] = measure_serving(dev, n_req=200, warmup=1)

    # ---------------------------------------------------------------- CPU baseline
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(args, cams)

    if rank == 0:
        clocks = clk.summary()
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_value / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(workload(args), parallelism=f"replicas x{world}"),
            "latency_ms": {"p50": pct(lat_value, 50), "p99": pct(lat_value, 99),
                           "note": f"submit-to-done per request with {args.slots} requests in flight"},
            "plain_per_call": {"value": plain_rps, "unit": UNIT, "value_at_p50": plain_rps_p50,
                               "p50_ms": pct(lat_plain, 50), "p99_ms": pct(lat_plain, 99), "requests": len(lat_plain),
                               "note": "one request at a time on one stream: preprocess, pair count read back, "
                                       "binning + blend, image copied to pinned host memory and waited for; "
                                       "workspaces kept between calls"},
            "served_over_plain": (e2e_value / plain_rps) if plain_rps else None,
            "served_over_plain_p50": (e2e_value / plain_rps_p50) if plain_rps_p50 else None,
            "served_over_plain_note": "e2e (served, every image copied to host) over the plain per-call leg with "
                                      "the same copy; _p50 uses the plain leg's median latency",
            "served_native": native,
            "e2e": {"value": e2e_value, "unit": UNIT,
                    "h2d_bytes_per_step": args.batch * 8 * (16 + 16 + 3 + 3 + 3 + 1),
                    "d2h_bytes_per_step": args.batch * 3 * args.width * args.height * 4,
                    "p50_ms": pct(lat_e2e, 50), "p99_ms": pct(lat_e2e, 99)},
            "roofline": {"kernel": "k_splat_blend", "bound": "hbm", "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "ms_per_launch": blend_ms, "n_pairs": n_pairs, "algorithmic_bytes": blend_bytes,
                         "bytes_formula": "40 P + 8 T + 12 px",
                         "frac_all_touched_bytes": blend_bytes_touched / (blend_ms * 1e-3) / 1e9 / peak,
                         "issue": issue_roof(warp_inst, blend_ms, clocks),
                         "l2": "flushed (256 MB write) before each timed launch",
                         "note": "the blend is bound by instruction issue, not HBM (see issue); frac_all_touched_bytes "
                                 "counts 48 P + 8 T + 20 px; traffic and warp instructions from the ncu capture of "
                                 "the same frame (profiles/splat_blend_1080p_1M.txt)"},
            "cpu_baseline": cpu,
            "clocks": clocks,
            "gpu_launches": int(launches),
            "rerenders": int(rerenders),
        }
        if extras:
            line.update(extras)
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()
    return 0


def _gpu_common():
    import torch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    return torch, torch.device("cuda", local), local


def measure_batched(dev, steps: int = 5, warmup: int = 3):
    """3 resident scenes (50k, 300k, 1.5M Gaussians) x 16 random cameras each,
    resolutions cycling 256x256 / 800x600 / 1920x1080, forward + backward of
    all 48 views per step: autotuned batch depth and blend block under CUDA graphs, against the
    plain per-view calls (forward, pair count read back, backward)."""
    import torch
    from differentiable_gaussian_mixture_renderer_b200 import scene as S
    from differentiable_gaussian_mixture_renderer_b200 import splat
    from differentiable_gaussian_mixture_renderer_b200.batch import BatchRenderer, autotune, chunks
    from differentiable_gaussian_mixture_renderer_b200.serving import GaussianScene, camera_struct
    sizes = {"s50k": 50_000, "s300k": 300_000, "s1500k": 1_500_000}
    res = [(256, 256), (800, 600), (1920, 1080)]
    scenes = {k: GaussianScene.from_numpy(S.make_scene(n, seed=i), dev) for i, (k, n) in enumerate(sizes.items())}
    views = []
    for j, k in enumerate(sizes):
        for v in range(16):
            w, h = res[v % 3]
            views.append((k, S.random_cameras(1, w, h, seed=100 * j + v)[0]))
    px = sum(c.width * c.height for _, c in views)
    r = BatchRenderer(scenes, dev)
    (best, block), timings = autotune(r, views, depths=(1, 4, 16, 48), backward=True, reps=2)
    plans = [r.capture(r.plan(c, backward=True), backward=True) for c in chunks(views, best)]
    gen = torch.Generator(device=dev).manual_seed(2)
    for p in plans:
        for g in p.grad_framebuffers:
            g.copy_(torch.randn(g.shape, device=dev, generator=gen))
    s0 = torch.cuda.current_stream(dev)

    def step():
        for p in plans:
            p.stream.wait_stream(s0)
            with torch.cuda.stream(p.stream):
                p.graph.replay()
        for p in plans:
            s0.wait_stream(p.stream)

    for _ in range(warmup):
        step()
    torch.cuda.synchronize(dev)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s0)
    for _ in range(steps):
        step()
    e1.record(s0)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / steps
    overflow = any(p.overflowed() for p in plans)
    # plain per-view calls, the reference's pattern (one view per call, P read back), workspaces kept
    ctx = splat.SplatContext(dev)
    lat = []
    for rep in range(2):  # the first pass grows the context's workspaces
        lat = []
        for k, (sid, cam) in enumerate(views):
            sc = scenes[sid]
            fb = plans[0].grad_framebuffers[0].new_empty((3, cam.height, cam.width))
            gfb = torch.ones_like(fb)
            torch.cuda.synchronize(dev)
            e0.record(s0)
            ctx.forward(sc.shs, sc.weights, sc.centroids, sc.scales, sc.rotations, camera_struct(cam), fb, sc.sh_degree)
            splat.splat_backward(ctx.frame(), gfb, sc.shs, sc.weights, sc.centroids, sc.scales, sc.rotations)
            e1.record(s0)
            e1.synchronize()
            lat.append(e0.elapsed_time(e1))
    plain_ms = sum(lat)
    return {"workload": "3 scenes (50k, 300k, 1.5M Gaussians) x 16 random cameras (r=2.5-4), resolutions cycling "
                        "256x256 / 800x600 / 1920x1080, forward + backward",
            "views": len(views), "megapixels_per_step": px / 1e6, "batch_depth": best, "blend_block": block, "ms_per_step": ms,
            "views_per_s": len(views) / (ms * 1e-3), "mpix_per_s": px / 1e6 / (ms * 1e-3),
            "autotune_ms": {f"depth {d}, blend block {b}x{b}": t for (d, b), t in timings.items()},
            "plain_per_view": {"views_per_s": len(views) / (plain_ms * 1e-3), "ms_per_step": plain_ms,
                               "note": "one view per call: forward (pair count read back) + backward, workspaces kept"},
            "batched_over_plain": plain_ms / ms, "pair_overflow": overflow, "graph_replays": steps * len(plans)}


def run_batched(args):
    """The batched workload (measure_batched) as its own JSON line."""
    torch, dev, local = _gpu_common()
    with ClockSampler(local) as clk:
        r = measure_batched(dev, steps=args.steps, warmup=args.warmup)
    line = {"metric": "batched views/s, forward+backward, 3 scenes x 16 views, mixed resolutions",
            "value": r["views_per_s"], "unit": "views/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": r.pop("workload"), "views": r["views"], "batch_depth": r["batch_depth"],
                       "l2": "working set of one step (~30M view-Gaussian slots) far above the 126 MB L2"},
            **r, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


MARCHER_PROFILE = "vol_marcher_c2_100k_512.txt"


def measure_marcher(dev, n_cams: int = 3, n: int = 100_000, W: int = 512, H: int = 512, seed_cams: int = 1):
    """vol_marcher forward + backward through the reference-facing binding
    (cpp_binding.forward / backward) at 100k Gaussians, 512x512, float32, one
    warm-up camera then ``n_cams`` timed ones; the forward also counts the
    march's work unit (bin fills, each 128 CDF evaluations) on the device."""
    import torch
    from differentiable_gaussian_mixture_renderer_b200 import _native as N
    from differentiable_gaussian_mixture_renderer_b200 import cpp_binding
    from differentiable_gaussian_mixture_renderer_b200 import scene as S
    sc = S.make_scene(n, seed=0)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float32).to(dev)
    ins = (t(sc.sh), t(sc.weights).reshape(-1, 1), t(sc.centroids), t(sc.scales), t(sc.rotations))
    cams = S.random_cameras(n_cams + 1, W, H, seed=seed_cams)
    G = torch.randn(3, H, W, device=dev, generator=torch.Generator(device=dev).manual_seed(2))
    bg = torch.zeros(3, device=dev)
    counter = torch.zeros(1, dtype=torch.int64, device=dev)
    fwd, bwd, fills, fwd_s, bwd_s = [], [], [], [], []
    store = cpp_binding.make_step_store(W, H, 4, device=dev)
    l0 = N.lib().dgmr_launch_count()
    for k, cam in enumerate(cams):
        v, p, c = t(cam.view), t(cam.proj), t(cam.campos)
        counter.zero_()
        e0, e1, e2, e3, e4 = (torch.cuda.Event(enable_timing=True) for _ in range(5))
        e0.record()
        cache = cpp_binding.forward(*ins, v, p, c, bg, W, H, cam.tan_fovx, cam.tan_fovy, 0, work_counter=counter)
        e1.record()
        cpp_binding.backward(*ins, v, p, c, bg, W, H, cam.tan_fovx, cam.tan_fovy, 0, G, cache)
        e2.record()
        # the same frame with the sample steps kept by the forward (vol_marcher.apply's default when memory allows)
        cache = cpp_binding.forward(*ins, v, p, c, bg, W, H, cam.tan_fovx, cam.tan_fovy, 0, step_store=store)
        e3.record()
        cpp_binding.backward(*ins, v, p, c, bg, W, H, cam.tan_fovx, cam.tan_fovy, 0, G, cache, step_store=store)
        e4.record()
        e4.synchronize()
        if k == 0:
            l0 = N.lib().dgmr_launch_count()
            continue
        fwd.append(e0.elapsed_time(e1))
        bwd.append(e1.elapsed_time(e2))
        fwd_s.append(e2.elapsed_time(e3))
        bwd_s.append(e3.elapsed_time(e4))
        fills.append(int(counter.item()))
    launches = N.lib().dgmr_launch_count() - l0
    fills_per_s = sum(fills) / (sum(fwd) * 1e-3)
    out = {"forward_ms": statistics.median(fwd), "backward_ms": statistics.median(bwd),
           "backward_over_forward": statistics.median(bwd) / statistics.median(fwd),
           "stored_steps": {"forward_ms": statistics.median(fwd_s), "backward_ms": statistics.median(bwd_s),
                            "backward_over_forward": statistics.median(bwd_s) / statistics.median(fwd_s),
                            "note": "forward keeps the first 4 large steps' samples of every ray, the backward reads "
                                    "them (vol_marcher.apply when the store fits 25 % of free memory)"},
           "bin_fills_per_frame": statistics.median(fills), "cdf_evaluations_per_s": 128 * fills_per_s,
           "gpu_launches": int(launches), "frames": len(fwd),
           "workload": f"vol_marcher forward + backward, {n} Gaussians (config-0 distribution), {W}x{H}, random "
                       "cameras r=2.5-4, through cpp_binding.forward/backward"}
    # FP32 roof of the forward: 148 SMs x 128 FP32 lanes per cycle, over the FP32 thread
    # instructions one bin fill takes (ncu count of the same frame / its fills)
    per_fill = profiled_value(MARCHER_PROFILE, "fp32_thread_inst_per_fill")
    if per_fill:
        peak = SMS * 128 * 1965e6 / per_fill
        out["roofline"] = {"kernel": "k_vm_march_warp", "bound": "fp32", "unit": "bin fills/s", "achieved": fills_per_s,
                           "peak": peak, "frac": fills_per_s / peak, "fp32_thread_inst_per_fill": per_fill,
                           "note": "forward call time (preprocess and binning included, < 2 % of it); peak at the "
                                   "1965 MHz maximum clock; FP32 instructions per fill from "
                                   f"profiles/{MARCHER_PROFILE}"}
    return out


def measure_marcher_batched(dev, n_views: int = 16, n: int = 100_000, W: int = 64, H: int = 64, reps: int = 2):
    """vol_marcher forward + backward of many small views (training-sized
    crops) of the c2 scene: one reference-facing call per view
    (cpp_binding.forward / backward) against one batched launch sequence
    (batch.BatchRenderer(kind="march"), dgmr_vm_batch_*).  CUDA events around
    the whole view set, one warm-up then the median of ``reps``."""
    import torch
    from differentiable_gaussian_mixture_renderer_b200 import cpp_binding
    from differentiable_gaussian_mixture_renderer_b200 import scene as S
    from differentiable_gaussian_mixture_renderer_b200.batch import BatchRenderer
    from differentiable_gaussian_mixture_renderer_b200.serving import GaussianScene
    sc = GaussianScene.from_numpy(S.make_scene(n, seed=0), dev)
    cams = S.random_cameras(n_views, W, H, seed=1)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float32).to(dev)
    gen = torch.Generator(device=dev).manual_seed(2)
    grads = [torch.randn(3, H, W, device=dev, generator=gen) for _ in cams]
    bg = torch.zeros(3, device=dev)

    def per_call():
        for cam, g in zip(cams, grads):
            args = (sc.shs, sc.weights.reshape(-1, 1), sc.centroids, sc.scales, sc.rotations, t(cam.view), t(cam.proj),
                    t(cam.campos), bg, W, H, cam.tan_fovx, cam.tan_fovy, 0)
            cpp_binding.backward(*args, g, cpp_binding.forward(*args))

    r = BatchRenderer({"c2": sc}, dev, kind="march")
    plan = r.plan([("c2", cam) for cam in cams], backward=True)
    for dst, g in zip(plan.grad_framebuffers, grads):
        dst.copy_(g)

    def batched():
        r.forward(plan)
        r.backward(plan)

    def timed(f):
        f()
        torch.cuda.synchronize()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            f()
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return statistics.median(ts)

    t_call, t_batch = timed(per_call), timed(batched)
    return {"per_call_ms": t_call, "batched_ms": t_batch, "views_per_s_per_call": 1e3 * n_views / t_call,
            "views_per_s_batched": 1e3 * n_views / t_batch, "batched_over_per_call": t_call / t_batch,
            "workload": f"vol_marcher forward + backward of {n_views} views of {W}x{H}, {n} Gaussians (the c2 scene), "
                        "one call per view vs one dgmr_vm_batch_* launch sequence"}


def measure_vol_raster(dev, n_cams: int = 3, n: int = 100_000, W: int = 512, H: int = 512):
    """vol_raster forward (the volume rasteriser, forward only) through
    vol_raster.forward at the c2 scene: 100k Gaussians, 512x512, one warm-up
    camera then ``n_cams`` timed ones (CUDA events around the call)."""
    import torch
    from differentiable_gaussian_mixture_renderer_b200 import scene as S
    from differentiable_gaussian_mixture_renderer_b200 import vol_raster
    sc = S.make_scene(n, seed=0)
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float32).to(dev)
    ins = (t(sc.sh), t(sc.weights), t(sc.centroids), t(sc.scales), t(sc.rotations))
    cams = S.random_cameras(n_cams + 1, W, H, seed=1)
    ms = []
    for k, cam in enumerate(cams):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        vol_raster.forward(*ins, t(cam.view), t(cam.proj), t(cam.campos), torch.zeros(3, device=dev), W, H,
                           cam.tan_fovx, cam.tan_fovy, 0)
        e1.record()
        e1.synchronize()
        if k:
            ms.append(e0.elapsed_time(e1))
    return {"forward_ms": statistics.median(ms), "mpix_per_s": W * H / 1e6 / (statistics.median(ms) * 1e-3),
            "workload": f"vol_raster forward, {n} Gaussians (config-0 distribution), {W}x{H}, random cameras r=2.5-4"}


def run_raster(args):
    """The vol_raster workload (measure_vol_raster) as its own JSON line."""
    torch, dev, local = _gpu_common()
    with ClockSampler(local) as clk:
        r = measure_vol_raster(dev, n_cams=max(args.steps, 1))
    line = {"metric": "vol_raster forward ms/frame, 100k Gaussians, 512x512", "value": r["forward_ms"], "unit": "ms",
            "n_gpus": 1, "steps": args.steps, "warmup": 1, "ms_per_step": r["forward_ms"], "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": r.pop("workload")}, **r, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


def run_marcher(args):
    """vol_marcher forward + backward through the reference-facing binding
    (cpp_binding.forward / backward): 100k Gaussians, 512x512, fp32."""
    torch, dev, local = _gpu_common()
    with ClockSampler(local) as clk:
        r = measure_marcher(dev, n_cams=max(args.steps, 1))
    ms = r["forward_ms"] + r["backward_ms"]
    line = {"metric": "vol_marcher forward+backward ms/frame, 100k Gaussians, 512x512", "value": ms, "unit": "ms",
            "n_gpus": 1, "steps": args.steps, "warmup": 1, "ms_per_step": ms, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": r.pop("workload")}, **r, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


def measure_serving(dev, n_req: int = 200, warmup: int = 1, rate: float = 200.0, native: bool = True):
    """8 resident scenes (100k-3M Gaussians, log-uniform), a Poisson request
    stream at ``rate`` req/s, resolutions drawn from 256^2 / 512^2 / 1280x720 /
    1920x1080, 20 % of requests also asking for the gradient against an N(0,1)
    image gradient.  The continuous-batching server, saturated (all requests
    queued at once) and on the Poisson arrivals, against a serial server that
    makes the plain per-request calls (preprocess, pair count read back,
    render, backward; workspaces kept) on the same arrival times.  ``native``:
    the C++ server (dgmr_server_*, NativeServer), else the Python one
    (ContinuousServer)."""
    import torch
    from differentiable_gaussian_mixture_renderer_b200 import scene as S
    from differentiable_gaussian_mixture_renderer_b200 import splat
    from differentiable_gaussian_mixture_renderer_b200.serving import (ContinuousServer, GaussianScene, NativeServer,
                                                                         ServeRequest, camera_struct)
    rng = np.random.default_rng(7)
    counts = np.exp(rng.uniform(np.log(1e5), np.log(3e6), size=8)).astype(int)
    scenes = {f"s{i}": GaussianScene.from_numpy(S.make_scene(int(n), seed=20 + i), dev) for i, n in enumerate(counts)}
    res = [(256, 256), (512, 512), (1280, 720), (1920, 1080)]
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=n_req))
    gen = torch.Generator(device=dev).manual_seed(3)

    def make_requests():
        out = []
        r2 = np.random.default_rng(11)
        for k in range(n_req):
            sid = f"s{int(r2.integers(8))}"
            w, h = res[int(r2.integers(4))]
            cam = S.random_cameras(1, w, h, seed=1000 + k)[0]
            bwd = bool(r2.uniform() < 0.2)
            g = torch.randn((3, h, w), device=dev, generator=gen) if bwd else None
            req = ServeRequest(sid, cam, backward=bwd, grad_image=g, arrival=float(arrivals[k]))
            # the client owns its output buffers (a pool in a real deployment): no allocation in the loop
            req.image = torch.empty((3, h, w), dtype=torch.float32, device=dev)
            if bwd:
                sc = scenes[sid]
                req.grads = tuple(torch.empty_like(t) for t in (sc.shs, sc.weights, sc.centroids, sc.scales,
                                                                 sc.rotations))
            out.append(req)
        return out

    server = (NativeServer if native else ContinuousServer)(scenes, dev, n_slots=4, max_batch=8)

    def counters():
        if native:
            st = server.stats()
            return st["rerenders"], st["reallocs"]
        return server.rerenders, server.reallocs

    def busy():
        if native:
            return server.poll() > 0
        return bool(server.queue or any(sl.batch for sl in server.slots))
    # warm-up: one pass over a request set of the same distribution (other cameras) learns every
    # (scene, resolution) pair capacity and grows the slots' workspaces to their steady size
    warm = make_requests()
    rw = np.random.default_rng(5)
    for r in warm:
        r.camera = S.random_cameras(1, r.camera.width, r.camera.height, seed=int(rw.integers(1 << 30)))[0]
    for _ in range(max(warmup, 1)):
        for r in warm:
            server.submit(r)
        server.drain()
    server.completed.clear()
    del warm

    def serve(reqs, poisson: bool):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        i = 0
        while True:
            now = time.perf_counter() - t0
            while i < len(reqs) and (not poisson or reqs[i].arrival <= now):
                reqs[i].arrival = reqs[i].arrival if poisson else 0.0
                server.submit(reqs[i])
                i += 1
            if not busy() and i >= len(reqs):
                break
            if not native:
                server.poll()
        torch.cuda.synchronize(dev)
        lat = [(r.t_done - t0 - r.arrival) * 1e3 for r in reqs]
        span = max(r.t_done for r in reqs) - t0
        return len(reqs) / span, lat

    def batch_log(reqs):
        if native:
            sizes = [r.batch_size for r in reqs]
            infl = [(r.t_done - r.t_launch) * 1e3 for r in reqs]
            return {"mean_requests": float(np.mean(sizes)), "in_flight_ms_p50": pct(infl, 50),
                    "in_flight_ms_p99": pct(infl, 99)}
        lg = server.log
        server.log = []
        if not lg:
            return {}
        inflight = [x[3] * 1e3 for x in lg]
        gpu = [x[4] for x in lg]
        return {"batches": len(lg), "mean_requests": float(np.mean([x[0] for x in lg])),
                "gpu_ms_p50": pct(gpu, 50), "gpu_ms_p99": pct(gpu, 99),
                "in_flight_ms_p50": pct(inflight, 50), "in_flight_ms_p99": pct(inflight, 99)}

    server.log = []
    reqs = make_requests()
    r0, a0 = counters()
    thr_poisson, lat_poisson = serve(reqs, True)
    batch_sizes = [r.batch_size for r in reqs]
    r1, a1 = counters()
    log_poisson = dict(batch_log(reqs), rerenders=r1 - r0, reallocs=a1 - a0)
    reqs = make_requests()
    r0, a0 = counters()
    thr_sat, lat_sat = serve(reqs, False)
    r1, a1 = counters()
    log_sat = dict(batch_log(reqs), rerenders=r1 - r0, reallocs=a1 - a0)
    if native:
        st = server.stats()
        budget_gb, peak_gb = st["hbm_budget_bytes"] / 1e9, st["hbm_peak_bytes"] / 1e9
        server.close()
    else:
        budget_gb, peak_gb = server.budget.budget / 1e9, server.budget.peak / 1e9
        server.drain()
    del server
    # plain per-request calls, one at a time, on the same arrival times
    reqs = make_requests()
    ctx = splat.SplatContext(dev)
    for r in reqs[:8]:  # grows the context's workspaces
        sc = scenes[r.scene_id]
        ctx.forward(sc.shs, sc.weights, sc.centroids, sc.scales, sc.rotations, camera_struct(r.camera), r.image,
                    sc.sh_degree)
    t_free = 0.0
    lat_plain, service = [], []
    for r in reqs:
        sc = scenes[r.scene_id]
        torch.cuda.synchronize(dev)
        t = time.perf_counter()
        ctx.forward(sc.shs, sc.weights, sc.centroids, sc.scales, sc.rotations, camera_struct(r.camera), r.image,
                    sc.sh_degree)
        if r.backward:
            splat.splat_backward(ctx.frame(), r.grad_image, sc.shs, sc.weights, sc.centroids, sc.scales, sc.rotations)
        torch.cuda.synchronize(dev)
        dt = time.perf_counter() - t
        service.append(dt)
        start = max(r.arrival, t_free)
        t_free = start + dt
        lat_plain.append((t_free - r.arrival) * 1e3)
    plain_thr = len(reqs) / sum(service)
    return {"workload": "8 scenes (100k-3M Gaussians, log-uniform, config-0 distribution), random cameras r=2.5-4, "
                        "resolutions from 256x256 / 512x512 / 1280x720 / 1920x1080, 20% gradient requests (N(0,1) "
                        "image gradient)",
            "scene_gaussians": [int(n) for n in counts], "requests": n_req, "slots": 4, "max_batch": 8,
            "saturation": {"requests_per_s": thr_sat, "p50_ms": pct(lat_sat, 50), "p99_ms": pct(lat_sat, 99),
                           "note": "all requests queued at t=0", "batches": log_sat},
            f"poisson_{int(rate)}": {"requests_per_s": thr_poisson, "p50_ms": pct(lat_poisson, 50),
                                     "p99_ms": pct(lat_poisson, 99), "mean_batch": float(np.mean(batch_sizes)),
                                     "batches": log_poisson},
            "plain_per_request": {"requests_per_s": plain_thr, "p50_ms": pct(lat_plain, 50),
                                  "p99_ms": pct(lat_plain, 99),
                                  "note": "serial per-request calls (workspaces kept) on the same Poisson arrivals"},
            "served_over_plain": thr_sat / plain_thr, "hbm_budget_gb": budget_gb, "hbm_peak_gb": peak_gb,
            "server": "C++ (dgmr_server_*)" if native else "Python (ContinuousServer)"}


def run_serving(args):
    """The serving workload (measure_serving) as its own JSON line."""
    torch, dev, local = _gpu_common()
    n_req = max(args.steps, 1) * 40
    with ClockSampler(local) as clk:
        r = measure_serving(dev, n_req=n_req, warmup=args.warmup, native=not args.python_server)
    thr = r["saturation"]["requests_per_s"]
    line = {"metric": "served requests/s + p50/p99 ms, continuous batching, 8 scenes, Poisson 200 req/s",
            "value": thr, "unit": "requests/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * n_req / thr / max(args.steps, 1), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": r.pop("workload"), "scene_gaussians": r.pop("scene_gaussians"),
                       "requests": n_req, "slots": 4, "max_batch": 8},
            **r, "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


def run_configs(args):
    """The parity configurations as per-call timings: splat forward 10k at
    256x256, splat forward + backward 200k at 1024x1024, vol_marcher forward +
    backward 100k at 512x512 -- each on the GPU (CUDA events around the calls,
    median over the cameras) and on the host through the oracle (a bounded
    sample: the first camera, or for the marcher a 128x128 frame of the same
    scene whose time is scaled by the pixel count)."""
    torch, dev, local = _gpu_common()
    from differentiable_gaussian_mixture_renderer_b200 import cpp_binding
    from differentiable_gaussian_mixture_renderer_b200 import scene as S
    from differentiable_gaussian_mixture_renderer_b200 import splat
    from oracle import oracle as O
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), dtype=torch.float32).to(dev)
    out = {}
    n_cams = args.warmup + args.steps

    def timed(fn):
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record()
        mid = fn(e1)
        e2.record()
        e2.synchronize()
        return e0.elapsed_time(e1), e1.elapsed_time(e2), mid

    for name, n, W, H, bwd in (("c0_splat_fwd_10k_256", 10_000, 256, 256, False),
                               ("c1_splat_fwd_bwd_200k_1024", 200_000, 1024, 1024, True)):
        sc = S.make_scene(n, seed=0, extent=2.0 if n == 200_000 else 1.0)
        ins = (t(sc.sh), t(sc.weights), t(sc.centroids), t(sc.scales), t(sc.rotations))
        cams = S.random_cameras(n_cams, W, H, seed=1)
        G = torch.randn(3, H, W, device=dev, generator=torch.Generator(device=dev).manual_seed(2))
        fw, bw = [], []
        for k, cam in enumerate(cams):
            def call(e_mid):
                fb, frame = splat.splat_forward(*ins, cam.view, cam.proj, cam.campos, (0.0, 0.0, 0.0), W, H, cam.tan_fovx,
                                                cam.tan_fovy, 0)
                e_mid.record()
                if bwd:
                    splat.splat_backward(frame, G, *ins)
                return frame
            a, b, _ = timed(call)
            if k >= args.warmup:
                fw.append(a)
                bw.append(b)
        r = {"gpu_fwd_ms": statistics.median(fw)}
        if bwd:
            r["gpu_bwd_ms"] = statistics.median(bw)
        if not args.no_cpu:
            c0 = time.perf_counter()
            ref = O.splat_forward(sc, cams[0])
            c1 = time.perf_counter()
            r["cpu_fwd_ms"] = (c1 - c0) * 1e3
            if bwd:
                O.splat_backward(sc, cams[0], ref, G.cpu().numpy())
                r["cpu_bwd_ms"] = (time.perf_counter() - c1) * 1e3
            r["cpu_cores"] = O.num_threads()
        out[name] = r

    n, W, H = 100_000, 512, 512
    sc = S.make_scene(n, seed=0)
    ins = (t(sc.sh), t(sc.weights).reshape(-1, 1), t(sc.centroids), t(sc.scales), t(sc.rotations))
    cams = S.random_cameras(n_cams, W, H, seed=1)
    G = torch.randn(3, H, W, device=dev, generator=torch.Generator(device=dev).manual_seed(2))
    bg = torch.zeros(3, device=dev)
    fw, bw = [], []
    for k, cam in enumerate(cams):
        v, pm, c = t(cam.view), t(cam.proj), t(cam.campos)

        def call(e_mid):
            cache = cpp_binding.forward(*ins, v, pm, c, bg, W, H, cam.tan_fovx, cam.tan_fovy, 0)
            e_mid.record()
            cpp_binding.backward(*ins, v, pm, c, bg, W, H, cam.tan_fovx, cam.tan_fovy, 0, G, cache)
            return cache
        a, b, _ = timed(call)
        if k >= args.warmup:
            fw.append(a)
            bw.append(b)
    r = {"gpu_fwd_ms": statistics.median(fw), "gpu_bwd_ms": statistics.median(bw)}
    if not args.no_cpu:
        small = S.make_camera(128, 128, eye=tuple(cams[0].campos.tolist()))
        c0 = time.perf_counter()
        cache = O.vm_forward(sc, small)
        c1 = time.perf_counter()
        O.vm_backward(sc, small, cache, np.zeros((3, 128, 128), np.float32) + 1.0)
        c2 = time.perf_counter()
        scale = (W * H) / (128 * 128)
        r.update(cpu_fwd_ms=(c1 - c0) * 1e3 * scale, cpu_bwd_ms=(c2 - c1) * 1e3 * scale, cpu_cores=O.num_threads(),
                 cpu_sample="one 128x128 frame of the same scene from the first camera's position, x16 for 512x512")
    out["c2_vol_marcher_fwd_bwd_100k_512"] = r
    line = {"metric": "per-call ms of the parity configurations", "value": out["c1_splat_fwd_bwd_200k_1024"]["gpu_fwd_ms"],
            "unit": "ms", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "higher_is_better": False,
            "dtype": "f32", "data": "synthetic", "config": {"workload": "c0 / c1 / c2 per-call timings"},
            "configs": out}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batched":
        return run_batched(args)
    if args.workload == "marcher":
        return run_marcher(args)
    if args.workload == "raster":
        return run_raster(args)
    if args.workload == "serving":
        return run_serving(args)
    if args.workload == "configs":
        return run_configs(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
