"""Multi-rank paths on CPU (gloo, world size 2): the split sweep and its gather.

sweep.shard_solve assigns instances to ranks (LPT), solves each rank's share
and all-gathers the R/T vectors so that every rank ends with the whole sweep
in instance order.  Here the solve is the oracle at 5x5 orders on small
stacks, so the test needs no GPU; the gathered results must equal the
single-process results bit for bit (same arithmetic, only moved).
"""
import os

import numpy as np
import pytest

from scattersim_b200 import samples, sweep

WORLD = 2


def small_sweep(count=7):
    inst = samples.sweep_instances(21, count=count, n=16, period=25.0)
    for i, it in enumerate(inst):
        it.orders = (3, 5)[i % 2]
        it.maps = it.maps[: 1 + i % 3]
    return inst


def oracle_solve(inst, idx):
    import torch
    from oracle import scattervolume as osv
    return [torch.from_numpy(osv.solve(inst[i].maps, osv.Params(**inst[i].params_kw()), keep=False).x) for i in idx]


def costs_sizes(inst):
    costs = [sweep.solve_cost(it.maps.shape[0], it.orders ** 2) for it in inst]
    sizes = [6 * it.orders ** 2 for it in inst]
    return costs, sizes


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        inst = small_sweep()
        costs, sizes = costs_sizes(inst)
        solved = []

        def fn(idx):
            solved.extend(idx)
            return oracle_solve(inst, idx)

        out = sweep.shard_solve(costs, sizes, fn, dist, "cpu")
        q.put((rank, sorted(solved), [o.numpy() for o in out]))
    finally:
        dist.destroy_process_group()


def run_ranks(target, world=WORLD):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29700 + os.getpid() % 1000
    procs = [ctx.Process(target=target, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = sorted([q.get(timeout=300) for _ in range(world)], key=lambda r: r[0])
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    return res


def test_split_sweep_gathers_every_instance_in_order():
    res = run_ranks(_worker)
    inst = small_sweep()
    costs, sizes = costs_sizes(inst)
    parts = sweep.assign_lpt(costs, WORLD)
    ref = [x.numpy() for x in oracle_solve(inst, range(len(inst)))]
    solved = []
    for rank, mine, out in res:
        assert mine == sorted(parts[rank])          # each rank solved exactly its share
        solved += mine
        assert len(out) == len(inst)
        for a, b in zip(out, ref):                  # every rank holds the whole sweep, in order
            assert a.shape == b.shape and np.array_equal(a, b)
    assert sorted(solved) == list(range(len(inst)))


def test_single_rank_shard_solve_is_local():
    inst = small_sweep(4)
    costs, sizes = costs_sizes(inst)
    out = sweep.shard_solve(costs, sizes, lambda idx: oracle_solve(inst, idx))
    ref = oracle_solve(inst, range(len(inst)))
    for a, b in zip(out, ref):
        assert np.array_equal(a.numpy(), b.numpy())


def test_gather_rejects_a_result_of_the_wrong_length():
    import torch

    class FakeDist:
        @staticmethod
        def is_initialized():
            return True

        @staticmethod
        def get_world_size():
            return 2

    with pytest.raises(ValueError):
        sweep.gather_results([0], [torch.zeros(3, dtype=torch.complex128)], [6, 6], [[0], [1]], FakeDist, "cpu")


# ---------------------------------------------------------------- one volume split by layers
LAYER_KW = dict(lambda_=0.6, size=(20.0, 20.0, 8.0), coef=(5, 5), ex=(1.0, 0.0), ey=(0.0, 0.0),
                direction=(0.17, 0.0, 0.98), external=True)


def layer_sample():
    return samples.sphere_volume(3, nxy=24, nz=7, size=(20.0, 20.0, 8.0))


def oracle_stages():
    import torch
    from oracle import scattervolume as osv
    smp = layer_sample()
    p = osv.Params(**LAYER_KW)

    def block(lb, le):
        P, G = osv.chain_block(smp, p, lb, le)
        return torch.from_numpy(P), (torch.from_numpy(G) if G is not None else None)

    def finish(g, gd):
        return torch.from_numpy(osv.boundary_from_chain(smp, p, g.numpy(), gd.numpy()))

    return block, (lambda a, b: a @ b), finish, 6 * 25, smp, p


def _layer_worker(rank, world, port, q):
    import datetime

    import torch.distributed as dist

    from scattersim_b200 import layersplit
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        block, mm, finish, n, smp, p = oracle_stages()
        x = layersplit.split_solve(smp.shape[0], block, mm, finish, n, dist, "cpu")
        q.put((rank, layersplit.layer_blocks(smp.shape[0], world)[rank], x.numpy()))
    finally:
        dist.destroy_process_group()


def test_layer_blocks_partition_in_order():
    from scattersim_b200 import layersplit
    for Z, w in [(7, 2), (32, 8), (5, 5), (9, 4)]:
        bl = layersplit.layer_blocks(Z, w)
        assert bl[0][0] == 0 and bl[-1][1] == Z
        assert all(a[1] == b[0] for a, b in zip(bl, bl[1:]))
        sizes = [e - b for b, e in bl]
        assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 1
    with pytest.raises(ValueError):
        layersplit.layer_blocks(2, 3)


@pytest.mark.parametrize("world", [2, 3])
def test_layer_split_equals_unsplit_chain(world):
    """Blocks on 2 and 3 gloo ranks, one exchange, ordered product on rank 0: the oracle's unsplit R/T."""
    from oracle import scattervolume as osv
    res = run_ranks(_layer_worker, world)
    _, _, _, _, smp, p = oracle_stages()
    ref = osv.solve(smp, p, keep=False).x
    for rank, blk, x in res:
        assert np.linalg.norm(x - ref) / np.linalg.norm(ref) < 1e-12, (rank, blk)


# ---------------------------------------------------------------- field grid split by z-planes
FIELD_COUNTS = (6, 5, 11)          # nx, ny, nz
FIELD_ORIGIN, FIELD_STEP = (-1.3, 0.4, -2.0), (0.37, 0.29, 0.41)


def field_table(seed=3):
    """A seeded wave table of three boundaries (incident, reflected and transmitted lists), unpacked."""
    from oracle import cw as ocw
    rng = np.random.default_rng(seed)

    def waves(n, down):
        kt = rng.uniform(-2.0, 2.0, (n, 2))
        kz = np.sqrt(40.0 - (kt ** 2).sum(1)) * (-1 if down else 1)
        k = np.c_[kt, kz].astype(np.complex128)
        E = rng.standard_normal((n, 3)) + 1j * rng.standard_normal((n, 3))
        return E, k
    PiE, Pik = waves(4, False)
    layers = []
    for z in (-1.0, 0.0, 1.5):
        PrE, Prk = waves(3, True)
        PtE, Ptk = waves(5, False)
        layers.append((z, PrE, Prk, PtE, Ptk))
    return ocw.unpack(PiE, Pik, layers)


def field_planes(WE, Wk, zl, b, e, lo, hi):
    """The oracle's evaluator on planes lo .. hi-1 of the test grid: (hi - lo, ny, nx, 3) (planes beyond the
    test grid's count follow the same spacing)."""
    import torch
    from oracle import cw as ocw
    nx, ny, _ = FIELD_COUNTS
    zz, yy, xx = np.meshgrid(FIELD_ORIGIN[2] + FIELD_STEP[2] * np.arange(lo, hi),
                             FIELD_ORIGIN[1] + FIELD_STEP[1] * np.arange(ny),
                             FIELD_ORIGIN[0] + FIELD_STEP[0] * np.arange(nx), indexing="ij")
    pts = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], -1)
    return torch.from_numpy(ocw.evaluate(pts, zl, b, e, WE, Wk).reshape(hi - lo, ny, nx, 3))


def _field_worker(rank, world, port, q, nz=FIELD_COUNTS[2]):
    import datetime

    import torch
    import torch.distributed as dist

    from scattersim_b200 import fieldsplit
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        zl, b, e, WE, Wk = field_table()
        # only rank 0 holds the table; the others receive it
        tE, tk = torch.from_numpy(WE.copy()), torch.from_numpy(Wk.copy())
        if rank != 0:
            tE.zero_()
            tk.zero_()
        fieldsplit.broadcast_tensors([tE, None, tk], dist)

        def fn(lo, hi):
            return field_planes(tE.numpy(), tk.numpy(), zl, b, e, lo, hi)
        counts = FIELD_COUNTS[:2] + (nz,)
        full = fieldsplit.split_grid(fn, counts, dist, "cpu")
        local, rng_ = fieldsplit.split_grid(fn, counts, dist, "cpu", gather=False)
        q.put((rank, full.numpy(), None if local is None else local.numpy(), rng_))
    finally:
        dist.destroy_process_group()


def test_plane_blocks_partition_in_order():
    from scattersim_b200 import fieldsplit
    for nz, w in [(11, 2), (64, 8), (5, 5), (3, 4), (0, 2)]:
        bl = fieldsplit.plane_blocks(nz, w)
        assert len(bl) == w and bl[0][0] == 0 and bl[-1][1] == nz
        assert all(a[1] == c[0] for a, c in zip(bl, bl[1:]))
        sizes = [hi - lo for lo, hi in bl]
        assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        fieldsplit.plane_blocks(4, 0)


@pytest.mark.parametrize("world", [2, 3])
def test_field_grid_split_equals_the_whole_grid(world):
    """z-slabs on 2 and 3 gloo ranks, the wave table broadcast from rank 0, the slabs all-gathered: every rank
    holds the single-process grid; without the gather each rank holds its own slab."""
    from scattersim_b200 import fieldsplit
    res = run_ranks(_field_worker, world)
    zl, b, e, WE, Wk = field_table()
    ref = field_planes(WE, Wk, zl, b, e, 0, FIELD_COUNTS[2]).numpy()
    blocks = fieldsplit.plane_blocks(FIELD_COUNTS[2], world)
    for rank, full, local, (lo, hi) in res:
        assert full.shape == ref.shape
        assert np.abs(full - ref).max() <= 1e-13 * np.abs(ref).max(), rank
        assert (lo, hi) == blocks[rank]
        assert np.abs(local - ref[lo:hi]).max() <= 1e-13 * np.abs(ref).max()


def test_field_grid_split_with_a_rank_holding_no_planes():
    """3 ranks, 2 planes: the last rank evaluates nothing yet takes part in the gather."""
    import functools
    from scattersim_b200 import fieldsplit
    res = run_ranks(functools.partial(_field_worker, nz=2), 3)
    zl, b, e, WE, Wk = field_table()
    ref = field_planes(WE, Wk, zl, b, e, 0, 2).numpy()
    for rank, full, local, (lo, hi) in res:
        assert np.abs(full - ref).max() <= 1e-13 * np.abs(ref).max(), rank
        assert (lo, hi) == fieldsplit.plane_blocks(2, 3)[rank]
        assert (local is None) == (hi == lo)


def test_slab_grid_assembles_blocks_in_order():
    from scattersim_b200 import fieldsplit
    zl, b, e, WE, Wk = field_table()
    ref = field_planes(WE, Wk, zl, b, e, 0, FIELD_COUNTS[2]).numpy()
    got = fieldsplit.slab_grid(lambda lo, hi: field_planes(WE, Wk, zl, b, e, lo, hi), FIELD_COUNTS,
                               fieldsplit.plane_blocks(FIELD_COUNTS[2], 4)).numpy()
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()
