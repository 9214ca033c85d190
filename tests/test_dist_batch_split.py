"""Batched systems over several GPUs are replicas: each rank solves its own
share of the systems (greedy balance by stored blocks, no communication) and
the job time is the slowest rank's. Checked on CPU with gloo ranks: every
system is solved exactly once, the shares are balanced, and the max-over-ranks
reduction of the timing is taken over all ranks."""
import os
import sys

import numpy as np
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _sizes():
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from monolis_b200 import problems
    sides = problems.batch_sides(512)
    return [7 * int(s) ** 3 for s in sides]  # ~ stored blocks of the 7-point systems


def test_split_covers_every_system_once_and_balances():
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    from monolis_b200 import partition
    nnz = _sizes()
    for world in (1, 2, 3, 4, 8):
        parts = partition.split_systems(nnz, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(nnz)))
        loads = [sum(nnz[i] for i in p) for p in parts]
        # greedy (LPT) bound: max load <= mean + largest system
        assert max(loads) <= sum(nnz) / world + max(nnz)
        if world > 1:
            assert max(loads) / (sum(nnz) / world) < 1.05  # many small systems: near-perfect balance


def _worker(rank, world, port, q):
    import datetime
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        if ROOT not in sys.path:
            sys.path.insert(0, ROOT)
        from monolis_b200 import partition
        nnz = _sizes()
        mine = partition.split_systems(nnz, world)[rank]
        # stand-in for the batched solve: time proportional to the share
        t = float(sum(nnz[i] for i in mine)) * 1e-9
        tt = torch.tensor([t], dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        q.put((rank, mine, t, tt.item()))
    finally:
        dist.destroy_process_group()


def test_ranks_take_disjoint_shares():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 34100 + (os.getpid() % 2000)
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    shares = [set(o[1]) for o in out]
    assert not (shares[0] & shares[1])
    assert len(shares[0] | shares[1]) == 512
    tmax = max(o[2] for o in out)
    assert all(abs(o[3] - tmax) == 0.0 for o in out)  # every rank holds the slowest rank's time
