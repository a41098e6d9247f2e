"""Sharding of independent solves across ranks.

Instances of a sweep (wavelengths x angles x samples, the workload the
reference runs as one scattervolume process per point, videomaker.py:61-74,
spectroscopy.py:66-91) are independent, so multi-GPU runs partition them with
no data-path collective.  The cost model is the dominant work of a solve:
layers x (2M)^3 for the eigensolves plus layers x (4M)^3 for the transfer
chain.  Assignment is greedy longest-processing-time first.
"""
from __future__ import annotations

import heapq


def solve_cost(layers: int, orders: int) -> float:
    """Relative device work of one solve with `layers` slices and M = orders."""
    n2 = 2 * orders
    return layers * (n2 ** 3 + 8.0 * n2 ** 3)


def assign_lpt(costs, world: int):
    """Greedy LPT: indices per rank, each rank's list in descending cost order."""
    if world <= 0:
        raise ValueError("world must be positive")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(world)]
    heapq.heapify(heap)
    out = [[] for _ in range(world)]
    for i in order:
        load, r = heapq.heappop(heap)
        out[r].append(i)
        heapq.heappush(heap, (load + costs[i], r))
    return out


def shard(costs, rank: int, world: int):
    """The instance indices rank `rank` of `world` solves."""
    return assign_lpt(costs, world)[rank]


def max_over_ranks(value: float, dist=None, device=None) -> float:
    """Max of a per-rank timing over the process group (identity without one)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
