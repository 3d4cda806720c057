"""Multi-process logic of bench.py on the CPU (gloo, world size 2).

One solve runs on one GPU; with N GPUs the benchmark runs N independent
replicas and reports the whole job's throughput from the slowest rank's time.
These tests run that aggregation as two gloo ranks, and check that the
reference arm under torchrun does its work on rank 0 only.
"""
import json
import os
import subprocess
import sys

import pytest
import torch.multiprocessing as tmp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    import bench
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        ms_local = 10.0 + 5.0 * rank          # rank 1 is the slow one
        ms = bench.max_over_ranks(ms_local, world, device="cpu")
        value = bench.replica_throughput(world, 1000, 7, ms)
        out[rank] = (ms, value)
    finally:
        dist.destroy_process_group()


def _free_port():
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_max_over_ranks_and_job_throughput():
    world = 2
    mgr = tmp.get_context("spawn").Manager()
    out = mgr.dict()
    tmp.spawn(_rank_main, args=(world, _free_port(), out), nprocs=world, join=True)
    # every rank sees the slowest rank's time; throughput counts all replicas' cells
    assert out[0][0] == out[1][0] == 15.0
    assert out[0][1] == out[1][1] == pytest.approx(2 * 1000 * 7 / 15e-3)


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(3.5, 1) == 3.5
    assert bench.replica_throughput(1, 100, 10, 1000.0) == pytest.approx(1000.0)


def test_reference_arm_runs_on_rank_zero_only():
    """A non-zero rank of `bench.py --impl reference` exits 0 at once and prints nothing."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "0"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""


def test_reference_arm_line():
    """Rank 0 of the reference arm prints the contract's JSON line (a tiny run)."""
    env = dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "0"],
                       env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] in ("reference", "port") and line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0
