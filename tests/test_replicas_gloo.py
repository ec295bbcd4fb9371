"""Replica plumbing on CPU with two gloo ranks: the max over ranks of a timed
region, the whole-job rate, and the ensemble member partition (every member
exactly once, balanced, identical on every rank)."""

import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from pygsquig_b200 import replicas as R


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        r, n = R.world()
        ms = R.max_over_ranks(10.0 * (rank + 1))
        costs = [R.member_cost(N, s) for N, s in [(128, 0)] * 48 + [(256, 1)] * 32 + [(512, 3)] * 16]
        mine = R.shard_members(costs, r, n)
        allparts = [None] * n
        dist.all_gather_object(allparts, mine)
        q.put((rank, r, n, ms, allparts))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    costs = [R.member_cost(N, s) for N, s in [(128, 0)] * 48 + [(256, 1)] * 32 + [(512, 3)] * 16]
    for rank, r, n, ms, parts in out:
        assert r == rank and n == world
        assert ms == 20.0  # the slower rank's time on both
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))  # each member exactly once
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) - min(loads) <= max(costs)
    assert out[0][4] == out[1][4]  # the same partition seen from both ranks


def test_job_rate_and_single_process():
    assert R.job_rate(50, 1000.0, 4) == pytest.approx(200.0)
    assert R.world() == (0, 1)
    assert R.max_over_ranks(3.5) == 3.5
    assert R.shard_members([1.0, 2.0, 3.0], 0, 1) == [0, 1, 2]
    with pytest.raises(ValueError):
        R.shard_members([1.0], 2, 2)
