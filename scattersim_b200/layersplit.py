"""One large volume solve split by layers over the ranks of a process group.

The transfer chain Gc_static = T_{Z-1} ... T_1 GC_0 (ScatterVolume.cpp:282-336)
is associative, so contiguous layer blocks can be solved independently: each
rank runs the Fourier, assembly and eigensolve stages of its block and forms
the ordered product of its block's transfer matrices
(sc_volume_chain_block); the products travel to rank 0 in one exchange
(point-to-point, NCCL over NVLink between GPUs), rank 0 multiplies them in
layer order, solves the boundary system (sc_volume_boundary_solve) and the
R/T vector is broadcast back.  The work per rank is its block's eigensolves
(the dominant stage); the exchange is one 4MF x 4MF matrix per rank.

``split_solve`` is the pattern with the stages as callables, so the same code
runs the GPU stages under NCCL and the oracle's CPU stages under gloo.
"""
from __future__ import annotations


def layer_blocks(Z: int, world: int):
    """Contiguous [begin, end) layer ranges, sizes differing by at most one, in layer order."""
    if world <= 0 or Z < world:
        raise ValueError(f"cannot split {Z} layers over {world} ranks")
    q, r = divmod(Z, world)
    out, b = [], 0
    for i in range(world):
        e = b + q + (1 if i < r else 0)
        out.append((b, e))
        b = e
    return out


def _flat_real(t):
    import torch
    return torch.view_as_real(t.contiguous()).reshape(-1)


def split_solve(Z, block_fn, matmul, finish_fn, x_size, dist=None, device=None):
    """Run one solve over the ranks of `dist` and return x = [R; T] on every rank.

    block_fn(lb, le) -> (P, GD0): the block's ordered transfer product (a
    complex128 tensor) and, for the block starting at layer 0, GD_0 (else
    None); matmul(A, B) -> A B; finish_fn(Gc_static, GD0) -> x (complex128,
    x_size values).  Without a process group everything runs locally.
    """
    import torch
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        P, GD0 = block_fn(0, Z)
        return finish_fn(P, GD0)
    rank, world = dist.get_rank(), dist.get_world_size()
    lb, le = layer_blocks(Z, world)[rank]
    P, GD0 = block_fn(lb, le)
    x = torch.empty(x_size, dtype=torch.complex128, device=device)
    if rank == 0:
        acc = P
        buf = torch.empty_like(P)
        for r in range(1, world):
            flat = _flat_real(buf)
            dist.recv(flat, src=r)
            buf = torch.view_as_complex(flat.reshape(-1, 2)).reshape(P.shape)
            acc = matmul(buf, acc)          # P_r (P_{r-1} ... P_0)
        x.copy_(finish_fn(acc, GD0).reshape(-1))
    else:
        dist.send(_flat_real(P), dst=0)
    flat = _flat_real(x)
    dist.broadcast(flat, src=0)
    return torch.view_as_complex(flat.reshape(-1, 2))
