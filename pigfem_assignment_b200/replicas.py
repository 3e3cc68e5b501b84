"""Host logic of the multi-GPU runs (one process per GPU).

A single RVE does not shard (its solve would need a halo exchange and a
reduction per Krylov dot), so `bench.py --gpus N` runs N replicas and times
them as the slowest rank.  A batch of independent RVEs shards with no
collective at all: each rank takes a share of the RVEs, balanced by element
count (longest processing time first), assembles and solves its share as its
own `pg_batch`, and only the timings and totals are reduced.
"""
from __future__ import annotations

import heapq
from typing import List, Sequence


def shard_rves(weights: Sequence[int], world: int) -> List[List[int]]:
    """Splits RVE indices over `world` ranks, heaviest first onto the least
    loaded rank; each rank's list is in ascending RVE order."""
    if world < 1:
        raise ValueError("world must be >= 1")
    heap = [(0, r) for r in range(world)]
    shards: List[List[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(weights)), key=lambda k: (-weights[k], k)):
        load, r = heapq.heappop(heap)
        shards[r].append(i)
        heapq.heappush(heap, (load + weights[i], r))
    return [sorted(s) for s in shards]


def _dist():
    import torch.distributed as dist
    return dist if dist.is_available() and dist.is_initialized() else None


def max_over_ranks(value: float, device=None) -> float:
    """The largest `value` over all ranks (the value itself without a process group)."""
    dist = _dist()
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    """The sum of `value` over all ranks (the value itself without a process group)."""
    dist = _dist()
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
