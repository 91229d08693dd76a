"""Placement of independent worlds on ranks (one process per GPU).

Batched worlds share nothing, so a multi-GPU batch is a partition of the world list: each
rank loads and steps its own worlds, and no data crosses between ranks while stepping.
The partition balances body counts, which set the per-step cost: greedy bin packing,
largest world first onto the least loaded rank (ties to the lower rank). Within a rank
the worlds keep their order in the batch.
"""
from __future__ import annotations

import heapq


def shard_worlds(sizes, world_size: int) -> list[list[int]]:
    """World indices per rank for worlds of the given body counts."""
    if world_size < 1:
        raise ValueError("world_size must be positive")
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    heap = [(0, r) for r in range(world_size)]
    shards: list[list[int]] = [[] for _ in range(world_size)]
    for i in order:
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + int(sizes[i]), r))
    return [sorted(s) for s in shards]


def max_over_ranks(value: float, device=None) -> float:
    """The largest value over all ranks of the default process group (the value itself when
    no group is initialised). Timings of a multi-GPU step are reported as this maximum."""
    import torch
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
