"""Sharding a batch over ranks (talus_b200.shard), CPU only.

* partition() gives contiguous, disjoint ranges that cover every body, none
  empty, with tet sums within a few percent of each other;
* a rank's bodies are exactly the corresponding bodies of the whole batch;
* two ranks on the gloo backend agree on the partition, and aggregate()
  returns the tets of both ranks and the slower rank's time, as bench.py
  reports them.
"""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from talus_b200 import shard


def test_partition_covers_every_body_once_and_balances():
    w = shard.tets_of(shard.batch_dims(1024)[0])
    for world in (1, 2, 3, 4, 8):
        parts = shard.partition(w, world)
        assert parts[0][0] == 0 and parts[-1][1] == w.size
        assert all(a < b for a, b in parts)
        assert all(parts[r][1] == parts[r + 1][0] for r in range(world - 1))
        sums = np.array([w[a:b].sum() for a, b in parts])
        assert sums.max() / sums.min() < 1.05, (world, sums)


def test_partition_edge_cases():
    assert shard.partition([5, 1, 1, 1], 4) == [(0, 1), (1, 2), (2, 3), (3, 4)]
    assert shard.partition([1, 1, 1, 100], 2) == [(0, 3), (3, 4)]
    with pytest.raises(ValueError):
        shard.partition([1], 2)


def test_rank_bodies_are_the_batch_bodies():
    from talus_b200 import mesh

    whole, wmats = mesh.batch_bodies(count=8, seed=5, lo=2, hi=4)
    part, pmats = shard.batch_bodies_range(3, 6, 8, seed=5, cells_lo=2, cells_hi=4)
    for a, b, ma, mb in zip(whole[3:6], part, wmats[3:6], pmats):
        assert np.array_equal(a.rest_positions, b.rest_positions)
        assert np.array_equal(a.tet_nodes, b.tet_nodes)
        assert ma[0] == mb[0]


def _rank(rank, world, port, out):
    import torch
    import torch.distributed as dist

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        dims = shard.batch_dims(64 * world, seed=3)
        lo, hi = shard.partition(shard.tets_of(dims), world)[rank]
        got = [None] * world
        dist.all_gather_object(got, (lo, hi))
        tets = int(shard.tets_of(dims)[lo:hi].sum())
        total, slowest = shard.aggregate(tets, 1.0 + rank, dist, "cpu")
        out.put((rank, got, tets, total, slowest))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_and_aggregate():
    world = 2
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    dims = shard.batch_dims(64 * world, seed=3)
    expected = shard.partition(shard.tets_of(dims), world)
    assert res[0][1] == res[1][1] == [tuple(x) for x in expected]
    total = sum(r[2] for r in res)
    assert total == int(shard.tets_of(dims).sum())
    assert all(r[3] == total and r[4] == 2.0 for r in res)
