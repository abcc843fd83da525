"""The multi-rank logic of bench.py (one replica per GPU) on gloo, world
size 2, on the CPU: the timed region is the slowest rank's and the value is
the whole job's throughput."""
import os
import sys

import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    sys.path.insert(0, ROOT)
    import datetime
    import bench
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    try:
        ms = bench.max_over_ranks(torch, 100.0 + 50.0 * rank, world, torch.device("cpu"))
        v = bench.replica_throughput(world, 2.0e12, ms)
        q.put((rank, ms, v))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 2000
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, ms, v in res:
        assert ms == 150.0                       # the slowest rank's time on every rank
        assert v == pytest.approx(2 * 2.0e12 / 0.150 / 1e12)


def test_single_rank_passthrough():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(torch, 12.5, 1, None) == 12.5
    assert bench.replica_throughput(1, 1.0e12, 1000.0) == pytest.approx(1.0)
