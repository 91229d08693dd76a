"""Multi-GPU path on the CPU: world sharding and max-over-ranks timing with two gloo ranks.

The single-world step runs as independent replicas (one per GPU); batched worlds are
partitioned across ranks with no collective on the data path, and every reported time is
the slowest rank's."""
from __future__ import annotations

import os
import socket
from datetime import timedelta

import numpy as np
import pytest

from avbd_demo3d_b200 import scenes
from avbd_demo3d_b200.sharding import max_over_ranks, shard_worlds


def test_shards_partition_the_worlds_and_balance_bodies():
    sizes = [sc.n_bodies for sc in scenes.batched_worlds(256, seed=3)]
    for ws in (1, 2, 3, 4, 8):
        shards = shard_worlds(sizes, ws)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(sizes)))
        assert all(s == sorted(s) for s in shards)
        loads = [sum(sizes[i] for i in s) for s in shards]
        # greedy largest-first: no rank exceeds the mean by more than one world
        assert max(loads) <= sum(sizes) / ws + max(sizes)


def test_shards_are_deterministic():
    sizes = [5, 9, 9, 3, 7, 1, 9]
    assert shard_worlds(sizes, 2) == shard_worlds(list(sizes), 2)
    assert shard_worlds(sizes, 1) == [list(range(7))]
    with pytest.raises(ValueError):
        shard_worlds(sizes, 0)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world_size, port, out):
    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world_size, timeout=timedelta(seconds=60))
    try:
        sizes = [sc.n_bodies for sc in scenes.batched_worlds(64, seed=3)]
        mine = shard_worlds(sizes, world_size)[rank]
        everyone = [None] * world_size
        dist.all_gather_object(everyone, mine)
        slowest = max_over_ranks(1.5 + rank)
        out.put((rank, everyone, slowest, len(sizes)))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_agree_on_shards_and_slowest_time():
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ws = 2
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, ws, port, q)) for r in range(ws)]
    for p in procs:
        p.start()
    results = [q.get(timeout=120) for _ in range(ws)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    results.sort()
    shards0 = results[0][1]
    for rank, shards, slowest, n in results:
        assert shards == shards0  # every rank derives the same placement
        assert slowest == pytest.approx(1.5 + ws - 1)
        assert sorted(i for s in shards for i in s) == list(range(n))
        assert not set(shards[0]) & set(shards[1])


def test_max_over_ranks_without_a_group():
    assert max_over_ranks(3.25) == 3.25
    assert np.isclose(max_over_ranks(np.float64(2.0)), 2.0)
