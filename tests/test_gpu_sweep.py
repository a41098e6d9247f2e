"""The batched sweep (sc_sweep_solve) against the CPU oracle and the plain GPU solve.

A sweep instance is one scattervolume --external solve (R/T only).  The
batched path computes the layer factors as matrix functions instead of
through eigenvectors, so parity is on the R/T vector: relative error <= 1e-9
against the oracle at sizes the oracle finishes in seconds, and against the
per-instance GPU path (itself pinned to the oracle) at the largest orders.
"""
import numpy as np
import pytest
import torch

from oracle import scattervolume as osv
from scattersim_b200 import _lib, samples, solver

pytestmark = pytest.mark.gpu

TOL = 1e-9


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def small_instances(count=8, orders=(7, 11), seed=3):
    inst = samples.sweep_instances(seed, count=count)
    for i, it in enumerate(inst):
        it.orders = orders[i % len(orders)]
    return inst


def run_sweep(ctx, inst, precision=_lib.SC_SWEEP_FP64):
    params = [solver.make_params(**it.params_kw()) for it in inst]
    smp = [torch.from_numpy(it.maps).cuda() for it in inst]
    return solver.sweep(ctx, params, smp, precision=precision)


def test_sweep_matches_oracle(ctx):
    inst = small_instances()
    res = run_sweep(ctx, inst)
    assert res.status == [0] * len(inst)
    for it, x in zip(inst, res.x):
        ref = osv.solve(it.maps, osv.Params(**it.params_kw()), keep=False).x
        assert rel(x.cpu().numpy(), ref) < TOL, (it.index, rel(x.cpu().numpy(), ref))


def test_sweep_uneven_shapes_and_single_layer(ctx):
    """Different slice shapes, one-layer stacks and non-square orders in one call."""
    rng = np.random.default_rng(11)
    cases = []
    for j, (shape, coef) in enumerate([((1, 40, 40), (5, 5)), ((3, 32, 24), (7, 5)), ((2, 48, 48), (5, 5)),
                                       ((1, 30, 36), (7, 5))]):
        smp = (1.0 + 0.5 * (rng.uniform(size=shape) > 0.5)).astype(np.complex128)
        kw = dict(lambda_=0.55 + 0.05 * j, size=(8.0, 8.0, 0.2 * shape[0]), coef=coef,
                  direction=(0.1 * j, 0.0, 1.0), ex=(1, 0), ey=(0, 0), external=True)
        cases.append((smp, kw))
    params = [solver.make_params(**kw) for _, kw in cases]
    res = solver.sweep(ctx, params, [torch.from_numpy(s).cuda() for s, _ in cases])
    for (smp, kw), x in zip(cases, res.x):
        ref = osv.solve(smp, osv.Params(**kw), keep=False).x
        assert rel(x.cpu().numpy(), ref) < TOL


def test_sweep_matches_plain_gpu_at_large_orders(ctx):
    """25x25 orders (n = 2500 per layer): batched path vs the per-instance path."""
    inst = samples.sweep_instances(5, count=4)
    for it in inst:
        it.orders = 25
        it.maps = it.maps[:4]
    res = run_sweep(ctx, inst)
    for it, x in zip(inst, res.x):
        p = solver.make_params(**it.params_kw())
        sol = solver.solve(ctx, p, torch.from_numpy(it.maps).cuda(), fields=False)
        assert rel(x.cpu().numpy(), sol.x.cpu().numpy()) < TOL


def test_sweep_energy_balance(ctx):
    """Lossless stacks conserve energy: sum |R|^2 Sz_top + |T|^2 Sz_bot equals the incident flux.

    The incident flux is |e|^2 cos(theta): the reference orthogonalises the
    polarisation against the direction without renormalising it
    (FourierWave.h:32-39), so an x-polarised wave at theta carries |e| = cos(theta).
    """
    inst = samples.sweep_instances(7, count=6)
    for i, it in enumerate(inst):
        it.orders = (15, 21)[i % 2]
    res = run_sweep(ctx, inst)
    for it, x, d in zip(inst, res.x, res.dims):
        p = osv.Params(**it.params_kw())
        _, e, dirv, k, ni, _, _, _, M, _ = osv.setup(it.maps, p)
        incident = float(np.sum(np.abs(e) ** 2) * np.real(dirv[2]))
        lat = osv.upwq_cal(M, p.size, dirv, k, ni)
        MF = M[0] * M[1]
        Sz0 = lat.Sz[0].ravel(order="F")
        Sz1 = lat.Sz[1].ravel(order="F")
        xv = x.cpu().numpy()
        R = (np.abs(xv[0:3 * MF].reshape(3, MF)) ** 2).sum(0) @ Sz0.real
        T = (np.abs(xv[3 * MF:].reshape(3, MF)) ** 2).sum(0) @ Sz1.real
        assert abs(R + T - incident) < 1e-9, (it.index, R + T, incident)


def test_sweep_per_instance_status(ctx):
    """A bad instance fails alone; the others are solved."""
    inst = small_instances(count=3)
    params = [solver.make_params(**it.params_kw()) for it in inst]
    params[1].lambda_ = -1.0
    smp = [torch.from_numpy(it.maps).cuda() for it in inst]
    # solver.sweep plans every instance first and would reject the bad one on
    # the host, so the call is made through the C ABI directly
    import ctypes
    n = len(inst)
    xs = [torch.zeros(6 * max(it.orders ** 2, 1), dtype=torch.complex128, device="cuda") for it in inst]
    P = (_lib.VolumeParams * n)(*params)
    S = (ctypes.c_void_p * n)(*[t.data_ptr() for t in smp])
    Z = (ctypes.c_int * n)(*[t.shape[0] for t in smp])
    S1 = (ctypes.c_int * n)(*[t.shape[1] for t in smp])
    S2 = (ctypes.c_int * n)(*[t.shape[2] for t in smp])
    X = (ctypes.c_void_p * n)(*[x.data_ptr() for x in xs])
    st = (ctypes.c_int * n)()
    rc = ctx.lib.sc_sweep_solve(ctx.handle, n, P, S, Z, S1, S2, X, 0, st, None)
    assert rc == _lib.SC_BADINPUT
    assert list(st) == [0, _lib.SC_BADINPUT, 0]
    for i in (0, 2):
        ref = osv.solve(inst[i].maps, osv.Params(**inst[i].params_kw()), keep=False).x
        assert rel(xs[i].cpu().numpy(), ref) < TOL


MIXED_TOL = 1e-8


@pytest.mark.parametrize("precision", [_lib.SC_SWEEP_MIXED, _lib.SC_SWEEP_SLICES(7)])
def test_sweep_mixed_matches_oracle(ctx, precision):
    """Autotuned mixed path, and every product forced onto the int8 tensor cores
    (7 digit slices): R/T within 1e-8 of the FP64 oracle."""
    inst = small_instances(count=6, seed=4)
    res = run_sweep(ctx, inst, precision=precision)
    for it, x in zip(inst, res.x):
        ref = osv.solve(it.maps, osv.Params(**it.params_kw()), keep=False).x
        assert rel(x.cpu().numpy(), ref) < MIXED_TOL, (it.index, rel(x.cpu().numpy(), ref))


def test_sweep_mixed_matches_fp64_at_large_orders(ctx):
    inst = samples.sweep_instances(6, count=4)
    for i, it in enumerate(inst):
        it.orders = (21, 25)[i % 2]
    fp = run_sweep(ctx, inst)
    for precision in (_lib.SC_SWEEP_MIXED, _lib.SC_SWEEP_SLICES(7)):
        mx = run_sweep(ctx, inst, precision=precision)
        for a, b in zip(mx.x, fp.x):
            assert rel(a.cpu().numpy(), b.cpu().numpy()) < MIXED_TOL


def test_sweep_slice_count_orders_error(ctx):
    """Each digit slice buys about 2^-7: the R/T error falls monotonically from 4 to 7 slices."""
    inst = small_instances(count=3, seed=8)
    fp = run_sweep(ctx, inst)
    errs = []
    for slices in (4, 5, 6, 7):
        sl = run_sweep(ctx, inst, precision=_lib.SC_SWEEP_SLICES(slices))
        errs.append(max(rel(a.cpu().numpy(), b.cpu().numpy()) for a, b in zip(sl.x, fp.x)))
    assert all(b < a for a, b in zip(errs, errs[1:])), errs
    assert errs[-1] < 1e-10 and errs[0] < 1e-3, errs
