"""World-size-2 gloo tests of the multi-rank host logic (no GPU): replicas take the max of the
per-rank step times, and the reference arm runs on rank 0 only."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    import datetime
    import sys

    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    dist.init_process_group("gloo", init_method="tcp://127.0.0.1:%d" % port, rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        got = bench.max_over_ranks([1.0 + rank, 10.0 - rank], dist, "cpu")
        q.put((rank, got))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_max_over_ranks_gloo():
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
    assert res[0] == [2.0, 10.0] and res[1] == [2.0, 10.0]


def test_max_over_ranks_single_process():
    import bench
    assert bench.max_over_ranks([3.0, 4.0]) == [3.0, 4.0]


def test_reference_arm_runs_on_rank0_only(monkeypatch, capsys):
    import bench

    class A:
        steps, warmup = 1, 0

    # a non-zero rank returns at once, prints nothing and touches no oracle
    bench.run_reference(A(), rank=1, world=2)
    assert capsys.readouterr().out == ""
