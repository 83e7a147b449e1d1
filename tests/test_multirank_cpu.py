"""The N>1 (replicas) path on CPU: gloo ranks, world size 2.

The renderer does not shard: each GPU serves its own requests against its own
resident scene, so the only cross-rank step is the timing aggregation of the
benchmark (slowest rank's time, sum of the ranks' renders).  These tests run
that aggregation over a real gloo process group, and the reference arm of the
benchmark under torchrun with two ranks (rank 0 prints one line, rank 1 exits
without work).
"""
from __future__ import annotations

import json
import os
import socket
import subprocess
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    sys.path.insert(0, ROOT)
    import bench

    def over(op):
        def reduce(x):
            t = torch.tensor([x], dtype=torch.float64)
            dist.all_reduce(t, op=op)
            return float(t.item())
        return reduce

    ms_local = [12.0, 20.0][rank]  # rank 1 is the slow one
    units_local = [8, 8][rank]
    ms, units, value = bench.replica_totals(ms_local, units_local, world, over(dist.ReduceOp.MAX),
                                            over(dist.ReduceOp.SUM))
    q.put((rank, ms, units, value))
    dist.barrier()
    dist.destroy_process_group()


def test_replica_totals_gloo_world2():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    res = sorted(q.get(timeout=5) for _ in range(2))
    for rank, ms, units, value in res:
        assert ms == 20.0  # max over ranks
        assert units == 16.0  # whole-job units
        assert value == pytest.approx(16 / 0.020)


def test_replica_totals_single_rank_identity():
    sys.path.insert(0, ROOT)
    import bench
    ms, units, value = bench.replica_totals(4.0, 10, 1, None, None)
    assert (ms, units) == (4.0, 10.0)
    assert value == pytest.approx(2500.0)


def test_reference_arm_torchrun_two_ranks():
    """bench.py --impl reference under torchrun: rank 0 alone runs and prints."""
    port = _free_port()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(port),
           os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
           "--gaussians", "2000", "--width", "64", "--height", "48", "--steps", "2", "--warmup", "1"]
    env = dict(os.environ, OMP_NUM_THREADS="2")
    out = subprocess.run(cmd, capture_output=True, text=True, timeout=300, env=env, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 1
    rec = json.loads(lines[0])
    assert rec["impl"] == "reference"
    assert rec["value"] > 0 and rec["unit"] == "renders/s"
    assert rec["cpu_baseline"]["kind"] == "port"
    assert rec["e2e"]["h2d_bytes_per_step"] == 0
