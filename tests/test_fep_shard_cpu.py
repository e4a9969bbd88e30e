"""Sharding of the batched FEP windows over ranks (host logic, no GPU): every box goes to exactly
one rank, the greedy assignment balances the estimated cost, and the one collective of the path
(summing disjoint per-window dU/dlambda slots over ranks) rebuilds the full vector on every rank
(world size 2, gloo)."""

import os
import socket

import numpy as np
import torch.multiprocessing as mp

from sponge_b200.fep import box_cost, shard_boxes


def test_shard_boxes_covers_and_balances():
    rng = np.random.default_rng(3)
    costs = list(rng.uniform(1.0, 16.0, 48))
    for world in (1, 2, 3, 4, 8):
        parts = shard_boxes(costs, world)
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(48))
        loads = [sum(costs[k] for k in p) for p in parts]
        # greedy largest-first: the spread is at most one box's cost
        assert max(loads) - min(loads) <= max(costs) + 1e-9


def test_box_cost_uses_atoms_and_grid():
    from sponge_b200 import systems
    a = systems.fep_box(500, 0.0, 1)
    b = systems.fep_box(2000, 0.0, 2)
    assert box_cost(b) > box_cost(a) > 0


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime
    import sys

    import torch
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    from sponge_b200.fep import shard_boxes
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        costs = [float(c) for c in range(1, 49)]
        mine = shard_boxes(costs, world)[rank]
        full = torch.zeros(48, dtype=torch.float64)
        full[torch.tensor(mine)] = torch.tensor([100.0 + k for k in mine], dtype=torch.float64)
        dist.all_reduce(full)
        q.put((rank, full.tolist()))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_dudl_gather_over_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = [100.0 + k for k in range(48)]
    assert res[0] == want and res[1] == want
