"""Query sharding across ranks (fasttree_b200/sharding.py): the plan on CPU, and the
multi-rank logic with two gloo ranks (every rank derives the same plan, the shards cover
the queries exactly once, the timing reduction takes the maximum)."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from fasttree_b200.sharding import max_over_ranks, shard_ranges


def test_even_ranges_cover_exactly_once():
    for num in (0, 1, 7, 100, 10_000_001):
        for world in (1, 2, 3, 8):
            r = shard_ranges(num, world)
            assert len(r) == world and r[0][0] == 0 and r[-1][1] == num
            assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
            sizes = [e - s for s, e in r]
            assert max(sizes) - min(sizes) <= 1


def test_cost_balanced_ranges():
    rng = np.random.default_rng(0)
    costs = rng.lognormal(0, 1.5, 50_000)
    for world in (2, 4, 8):
        r = shard_ranges(len(costs), world, costs)
        assert r[0][0] == 0 and r[-1][1] == len(costs)
        assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
        shares = [costs[s:e].sum() for s, e in r]
        # each share within one query's cost of the ideal
        assert max(abs(x - costs.sum() / world) for x in shares) <= costs.max() + 1e-9


def test_degenerate_costs_and_errors():
    assert shard_ranges(5, 2, np.zeros(5)) == shard_ranges(5, 2)
    r = shard_ranges(6, 3, [0, 0, 10, 0, 0, 0])
    assert r[0][0] == 0 and r[-1][1] == 6 and all(s <= e for s, e in r)
    with pytest.raises(ValueError):
        shard_ranges(3, 0)
    with pytest.raises(ValueError):
        shard_ranges(3, 2, [1, -1, 1])
    with pytest.raises(ValueError):
        shard_ranges(3, 2, [1, 1])


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, costs, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        plan = shard_ranges(len(costs), world, costs)
        # every rank must hold the same plan: gather all of them
        mine = torch.tensor([v for se in plan for v in se], dtype=torch.int64)
        all_plans = [torch.zeros_like(mine) for _ in range(world)]
        dist.all_gather(all_plans, mine)
        start, end = plan[rank]
        # each rank "answers" its queries: mark them, then sum the marks over ranks
        marks = torch.zeros(len(costs), dtype=torch.int32)
        marks[start:end] = 1
        dist.all_reduce(marks)
        t = max_over_ranks(10.0 * (rank + 1))
        out[rank] = (all(torch.equal(p, mine) for p in all_plans), bool(torch.all(marks == 1)), t)
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_and_cover():
    costs = np.random.default_rng(3).lognormal(0, 1, 10_000)
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_worker, args=(2, _free_port(), costs, out), nprocs=2, join=True)
    assert out[0] == (True, True, 20.0) and out[1] == (True, True, 20.0)


def _bytes_worker(rank, world, port, out):
    from fasttree_b200.sharding import broadcast_bytes
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        data = torch.from_numpy(np.random.default_rng(4).integers(0, 256, 100_003, dtype=np.uint8))
        got = broadcast_bytes(data if rank == 1 else None, 1)
        out[rank] = bool(torch.equal(got, data))
    finally:
        dist.destroy_process_group()


def test_broadcast_bytes_two_gloo_ranks():
    """The byte broadcast under broadcast_tree: a buffer of any size from a chosen rank."""
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_bytes_worker, args=(2, _free_port(), out), nprocs=2, start_method="spawn")
        assert out[0] and out[1]
