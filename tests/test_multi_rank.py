"""bench.py's multi-GPU plumbing on CPU ranks (gloo, world size 2): the path
runs N independent replicas, so the only cross-rank steps are the barrier and
the max-over-ranks timing; whole-job throughput is every rank's updates over
the slowest rank's time.  The reference arm runs on rank 0 alone."""

from __future__ import annotations

import datetime
import json
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

from tests.conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        bench._barrier(dist)
        dt_local = 1.0 + rank  # rank 1 is the slow one
        value, dt = bench.replica_throughput(dist, 1000, dt_local)
        out[rank] = (value, dt)
    finally:
        dist.destroy_process_group()


def test_replica_throughput_uses_the_slowest_rank():
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(120)
            assert p.exitcode == 0
        for r in range(2):
            value, dt = out[r]
            assert dt == 2.0
            assert value == 2 * 1000 / 2.0


def test_single_process_needs_no_group():
    sys.path.insert(0, str(ROOT))
    import bench

    assert bench.replica_throughput(None, 500, 0.5) == (1000.0, 0.5)


def test_reference_arm_runs_on_rank_zero_only():
    """Rank 1 of the reference arm exits 0 at once, printing nothing."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "0"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""


def test_extra_workloads_refuse_several_ranks():
    env = dict(os.environ, RANK="0", WORLD_SIZE="2", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--workload", "disk_oh65"], env=env,
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert "unavailable" in line
