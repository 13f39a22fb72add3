"""Host-side multi-GPU planning for the B200 path (no data-path collectives).

One field's 3D FFT does not shard without an all-to-all transpose, so N GPUs
run N independent fields (replicas) or split an ensemble's independent members.
This module holds the host logic: longest-processing-time (LPT) packing of
members onto ranks and the max-over-ranks reduction used for timing.
"""
from __future__ import annotations

import heapq
import math


def member_cost(n) -> float:
    """Work of one member per step, proportional to N log N of its 3D transform."""
    cells = int(n[0]) * int(n[1]) * int(n[2])
    return cells * math.log2(max(cells, 2))


def lpt_partition(costs, world_size: int):
    """Assign items (by cost) to `world_size` ranks, largest first onto the least
    loaded rank.  Returns (list of index lists, list of loads).  Deterministic:
    ties go to the lower rank / lower index."""
    if world_size < 1:
        raise ValueError("world_size must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world_size)]
    parts = [[] for _ in range(world_size)]
    for i in order:
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    loads = [sum(costs[i] for i in p) for p in parts]
    for p in parts:
        p.sort()
    return parts, loads


def members_for_rank(members, rank: int, world_size: int):
    """The ensemble members (dicts with key "n") that rank `rank` runs."""
    parts, _ = lpt_partition([member_cost(m["n"]) for m in members], world_size)
    return [members[i] for i in parts[rank]]


def max_over_ranks(value: float, device=None) -> float:
    """Maximum of `value` over all ranks of the default process group (identity
    without one).  Every rank must call it at the same point."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float, device=None) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
