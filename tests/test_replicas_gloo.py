"""The multi-GPU form is replicas only: every rank renders its own views and
the only collective is the max-reduction of the timed seconds.  These tests
run that path as two gloo processes on the CPU."""
import json
import os
import socket
import subprocess
import sys

import pytest

torch = pytest.importorskip("torch")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    from datetime import timedelta

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=timedelta(seconds=60))
    try:
        slowest = bench.slowest_rank_seconds(1.5 + rank, device="cpu")
        q.put((rank, slowest))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_slowest_rank_seconds_over_two_gloo_ranks():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    got = dict(q.get(timeout=10) for _ in range(2))
    assert got == {0: 2.5, 1: 2.5}   # every rank reports the slowest rank's time


def test_single_process_needs_no_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.slowest_rank_seconds(0.25, device="cpu") == 0.25


def test_reference_arm_prints_on_rank_zero_only():
    """Under torchrun the reference arm runs on rank 0; other ranks exit 0 without work."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                         env=env, capture_output=True, text=True, timeout=300)
    assert out.returncode == 0
    assert out.stdout.strip() == ""


def test_serving_reference_arm_is_unavailable_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--workload",
                          "serving"], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0
    line = json.loads(out.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and "unavailable" in line
