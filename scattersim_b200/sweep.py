"""Splitting one sweep of independent solves across ranks (one process per GPU).

Instances of a sweep (wavelengths x angles x samples, the workload the
reference runs as one scattervolume process per point, videomaker.py:61-74,
spectroscopy.py:66-91) are independent, so a multi-GPU run partitions them:
each rank solves its share with the batched path and the R/T vectors are
gathered at the end (the only collective).  Assignment is greedy
longest-processing-time first over a cost model of the batched path.

``shard_solve`` is the whole pattern: assignment, the rank's solve, and an
all-gather that returns every instance's result, in instance order, on every
rank.  The solve is a callable, so the same code runs the GPU sweep under NCCL
and a CPU solve under gloo.
"""
from __future__ import annotations

import heapq


def solve_cost(layers: int, orders: int) -> float:
    """Relative device work of one batched-path solve with `layers` slices and M = orders Fourier orders.

    Per layer the batched path forms its layer factor from about twelve
    products of order 2M (Taylor terms, squarings, the factored finish) and
    applies it in the chain by four products of (2M)^2 3M; the boundary
    system of order 6M is one LU, about nine (2M)^3 products.
    """
    n2 = 2.0 * orders
    return (12.0 * layers + 9.0) * n2 ** 3


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


def gather_results(mine, local, sizes, parts, dist=None, device=None):
    """All-gather the per-instance complex128 vectors of every rank.

    mine: this rank's instance indices; local: its result vectors in that
    order; sizes: the length of every instance's vector (known to all ranks);
    parts: every rank's index list (the assignment).  Each rank packs its
    vectors back to back as interleaved (re, im) float64, padded to the
    longest rank's length, so one all-gather of equal-size buffers moves
    everything; the result is the list of all instances' vectors in instance
    order, on every rank (on `device`).
    """
    import torch
    n = len(sizes)
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        out = [None] * n
        for i, v in zip(mine, local):
            out[i] = v
        return out
    world = dist.get_world_size()
    lengths = [2 * sum(sizes[i] for i in p) for p in parts]
    cap = max(max(lengths), 1)
    buf = torch.zeros(cap, dtype=torch.float64, device=device)
    off = 0
    for i, v in zip(mine, local):
        if v.numel() != sizes[i]:
            raise ValueError(f"instance {i}: result has {v.numel()} values, expected {sizes[i]}")
        buf[off:off + 2 * sizes[i]] = torch.view_as_real(v.reshape(-1).to(device)).reshape(-1)
        off += 2 * sizes[i]
    bufs = [torch.empty(cap, dtype=torch.float64, device=device) for _ in range(world)]
    dist.all_gather(bufs, buf)
    out = [None] * n
    for r, p in enumerate(parts):
        off = 0
        for i in p:
            out[i] = torch.view_as_complex(bufs[r][off:off + 2 * sizes[i]].reshape(-1, 2))
            off += 2 * sizes[i]
    return out


def shard_solve(costs, sizes, solve_fn, dist=None, device=None):
    """Solve a sweep split across the ranks of `dist` and return every result on every rank.

    costs: per-instance relative cost (solve_cost); sizes: per-instance result
    length (6 MF for R/T); solve_fn(indices) -> list of complex128 vectors for
    those instances, in that order.  Without a process group it solves
    everything locally.
    """
    if dist is None or not dist.is_initialized():
        rank, world = 0, 1
    else:
        rank, world = dist.get_rank(), dist.get_world_size()
    parts = assign_lpt(costs, world)
    mine = parts[rank]
    local = solve_fn(mine) if mine else []
    return gather_results(mine, local, sizes, parts, dist, device)
