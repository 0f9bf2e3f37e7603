"""N>1 harness of bench.py on CPU: two gloo ranks.

The path runs as independent replicas (one per GPU, no collective on the data
path); what the ranks share is the timing rule: every rank's timed region is
bracketed by a barrier, the reported time is the max over ranks, and the value
is the whole job's pairs over that time.  These tests run that host logic with
world_size 2 over gloo on 127.0.0.1, plus the reference arm's rank rule (rank 0
alone runs and prints; the others exit 0 without work).
"""
import os
import socket
import subprocess
import sys

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import bench
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        dist.barrier()
        # rank r "took" (r + 1) * 1.5 ms; every rank must report the slowest
        ms = bench.max_over_ranks(dist, (rank + 1) * 1.5, "cpu")
        e2e = bench.max_over_ranks(dist, 0.25 if rank == 0 else 0.5, "cpu")
        value = bench.replica_value(world, 2000 * 2000, ms / 1e3)
        dist.barrier()
        q.put((rank, ms, e2e, value))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_world2():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    out.sort()
    for rank, ms, e2e, value in out:
        assert ms == pytest.approx(3.0)
        assert e2e == pytest.approx(0.5)
        # both replicas' 2000^2 cells over the slowest rank's 3 ms
        assert value == pytest.approx(2 * 2000 * 2000 / 3e-3)


def test_max_over_ranks_single_process():
    import bench
    assert bench.max_over_ranks(None, 1.25, "cpu") == 1.25
    assert bench.replica_value(1, 100, 0.5) == 200


def test_reference_arm_nonzero_rank_exits_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
