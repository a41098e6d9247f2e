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
