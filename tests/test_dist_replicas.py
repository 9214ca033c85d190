"""The multi-GPU path of bench.py is independent replicas: each rank solves
its own system and the reported time is the maximum over ranks. Checked here
with two gloo processes on the CPU (no GPU): the helper returns the slowest
rank's value on every rank."""
import os
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        local = [0.5, 1.25][rank]
        got = bench.max_over_ranks(local, world, device="cpu")
        q.put((rank, got))
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_gloo_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + (os.getpid() % 2000)
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = dict(q.get(timeout=5) for _ in range(2))
    assert res == {0: 1.25, 1: 1.25}


def test_max_over_ranks_single_rank_is_identity():
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(0.75, 1) == 0.75
