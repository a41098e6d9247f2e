"""The field on a grid split by z-planes over the ranks of a process group.

The field at a grid point (the evaluator sum of gpuEvaluator.cu:28-68, which
sc_volume_field_grid forms for whole grids) depends only on that point and on
the solution, so the planes of a grid split into contiguous z-slabs, one per
rank.  Every rank needs the whole solution the grid is evaluated from (the R/T
vector and the layers' eigenvalues and mode fields): rank 0 broadcasts it
once (NCCL over NVLink between GPUs), each rank evaluates its slab, and the
slabs are all-gathered in plane order -- or left where they are, for a
consumer that writes or reduces each slab itself.  Per rank the work is its
share of the planes; the traffic is the solution once plus the grid once.

``split_grid`` takes the evaluation as a callable of a plane range, so the
same code runs the GPU evaluator under NCCL and the oracle's evaluator under
gloo; ``slab_grid`` evaluates given blocks one after the other on one device,
which is how one GPU checks the slab arithmetic of a split without waiting on
other ranks.
"""
from __future__ import annotations


def plane_blocks(nz: int, world: int):
    """Contiguous [begin, end) plane ranges in plane order, sizes differing by at most one (a rank beyond the
    plane count gets an empty range)."""
    if world <= 0 or nz < 0:
        raise ValueError(f"cannot split {nz} planes over {world} ranks")
    q, r = divmod(nz, world)
    out, b = [], 0
    for i in range(world):
        e = b + q + (1 if i < r else 0)
        out.append((b, e))
        b = e
    return out


def _flat(t):
    """A flat real view of a contiguous tensor (complex as interleaved reals), for the collectives."""
    import torch
    return (torch.view_as_real(t) if t.is_complex() else t).reshape(-1)


def broadcast_tensors(tensors, dist, src: int = 0):
    """Broadcast each tensor in place from rank `src` (every rank passes tensors of the same shapes and
    dtypes, contiguous; None entries are skipped on every rank alike)."""
    for t in tensors:
        if t is None:
            continue
        if not t.is_contiguous():
            raise ValueError("broadcast_tensors needs contiguous tensors")
        dist.broadcast(_flat(t), src=src)


def slab_grid(grid_fn, counts, blocks):
    """The grid assembled from the given plane blocks evaluated in turn: grid_fn(b, e) -> (e - b, ny, nx, 3)."""
    import torch
    parts = [grid_fn(b, e) for b, e in blocks if e > b]
    return torch.cat(parts, 0)


def split_grid(grid_fn, counts, dist=None, device=None, dtype=None, gather: bool = True):
    """Evaluate the grid of `counts` = (nx, ny, nz) over the ranks of `dist`.

    grid_fn(b, e) -> tensor (e - b, ny, nx, 3): the field on planes b .. e-1.
    With gather, every rank returns the whole (nz, ny, nx, 3) grid; without,
    each returns (its slab or None, (b, e)).  Without a process group (or with
    one rank) everything runs locally.
    """
    import torch
    nx, ny, nz = (int(c) for c in counts)
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        full = grid_fn(0, nz)
        return full if gather else (full, (0, nz))
    rank, world = dist.get_rank(), dist.get_world_size()
    blocks = plane_blocks(nz, world)
    b, e = blocks[rank]
    local = grid_fn(b, e) if e > b else None
    if not gather:
        return local, (b, e)
    dtype = dtype or (local.dtype if local is not None else torch.complex128)
    cap = max(hi - lo for lo, hi in blocks)
    buf = torch.zeros((cap, ny, nx, 3), dtype=dtype, device=device)
    if local is not None:
        buf[: e - b].copy_(local)
    parts = [torch.empty_like(buf) for _ in range(world)]
    dist.all_gather([_flat(p) for p in parts], _flat(buf))
    return torch.cat([parts[r][: hi - lo] for r, (lo, hi) in enumerate(blocks)], 0)
