"""The field evaluator on the reference's own coupled-wave data (fixture subsample).

The plane-wave sum of gpuEvaluator.cu:28-68 is checked in float64 (bar 1e-12)
and in float32 with float64 phase reduction (bar 1e-5 relative, the
reference's own evaluator sums in float32), through both the device entry
point and the host-buffer gpu_initialize / gpu_cw_evaluate shim.
"""
import ctypes
import os

import numpy as np
import pytest
import torch

from oracle import cw as ocw
from scattersim_b200 import samples, solver

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def fixture_table(tag):
    fx = np.load(os.path.join(GOLD, "cw_fixtures.npz"))
    layers = []
    for l in range(len(fx[f"{tag}_z"])):
        layers.append((float(fx[f"{tag}_z"][l]), ocw.get_e0_tira(fx[f"{tag}_L{l}_Pr_E"], fx[f"{tag}_L{l}_Pr_k"]),
                       fx[f"{tag}_L{l}_Pr_k"], ocw.get_e0_tira(fx[f"{tag}_L{l}_Pt_E"], fx[f"{tag}_L{l}_Pt_k"]),
                       fx[f"{tag}_L{l}_Pt_k"]))
    return ocw.unpack(ocw.get_e0_tira(fx[f"{tag}_Pi_E"], fx[f"{tag}_Pi_k"]), fx[f"{tag}_Pi_k"], layers)


@pytest.mark.parametrize("tag", ["psf", "acw"])
@pytest.mark.parametrize("precision,tol", [(0, 1e-12), (1, 1e-5)])
def test_evaluate_reference_waves(ctx, tag, precision, tol):
    from scattersim_b200.solver import evaluate
    zl, b, e, WE, Wk = fixture_table(tag)
    ext = 8.0
    pts = np.concatenate([ocw.slice_points(1, (0, 0, 0), ext, 40, 0.3), ocw.slice_points(2, (0, 0, 0), ext, 16, zl[0] + 0.5)])
    ref = ocw.evaluate(pts, zl, b, e, WE, Wk)
    got = evaluate(ctx, torch.from_numpy(WE).cuda(), torch.from_numpy(Wk).cuda(), zl, b, e,
                   torch.from_numpy(pts).cuda(), precision=precision).cpu().numpy()
    err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
    assert err < tol, err


def test_gpu_cw_evaluate_shim_matches_float32_sum(ctx):
    """gpu_initialize + gpu_cw_evaluate with host buffers (UnpackedWave<float> table)."""
    from scattersim_b200 import _lib
    lib = _lib.load()
    zl, b, e, WE, Wk = fixture_table("acw")
    W = np.empty((len(WE), 6), dtype=np.complex64)
    W[:, 0:3] = WE
    W[:, 3:6] = Wk
    zf = zl.astype(np.float32)
    layers = len(zl)
    _lib.check(lib.sc_gpu_initialize(layers, zf.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                     b.astype(np.int32).ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                     e.astype(np.int32).ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                     W.ctypes.data_as(ctypes.c_void_p), len(W), 0))
    N, ext = 32, 10.0
    d = ext / (N - 1)
    x0 = y0 = z0 = -ext / 2
    outs = [np.zeros((N, N, 3), dtype=np.complex64) for _ in range(3)]
    _lib.check(lib.sc_gpu_cw_evaluate(*[o.ctypes.data_as(ctypes.c_void_p) for o in outs], x0, y0, z0, 0.25, -0.5,
                                      1.5, d, N, 0))
    E_xy, E_xz, E_yz = outs
    # reference float32 sums at the same float32 grid points (x-z slice at y = -0.5)
    i = np.arange(N, dtype=np.float32)
    zz, xx = np.meshgrid(np.float32(z0) + np.float32(d) * i, np.float32(x0) + np.float32(d) * i, indexing="ij")
    pts = np.stack([xx.ravel(), np.full(N * N, np.float32(-0.5)), zz.ravel()], -1).astype(np.float64)
    ref = ocw.evaluate(pts, zf.astype(np.float64), b, e, W[:, 0:3].astype(np.complex128),
                       W[:, 3:6].astype(np.complex128), eps=0.001)
    got = E_xz.reshape(-1, 3)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-5


# ---------------------------------------------------------------- factorised grid evaluator
def _grid_points(origin, step, counts):
    nx, ny, nz = counts
    zz, yy, xx = np.meshgrid(origin[2] + step[2] * np.arange(nz), origin[1] + step[1] * np.arange(ny),
                             origin[0] + step[0] * np.arange(nx), indexing="ij")
    return np.stack([xx.ravel(), yy.ravel(), zz.ravel()], -1)


@pytest.mark.parametrize("kw,counts", [
    (dict(lambda_=0.6, size=(20, 20, 8), coef=(7, 5), direction=(0.17, 0.05, 0.98), ex=(1, 0), ey=(0, 0)),
     (17, 9, 23)),
    (dict(lambda_=0.55, size=(20, 20, 8), coef=(5, 5), external=True), (12, 1, 31)),
    (dict(lambda_=0.6, size=(20, 20, 8), coef=(9, 9), npz=True, kappa=0.02), (8, 6, 40)),
])
def test_field_grid_equals_direct_sum(ctx, kw, counts):
    """sc_volume_field_grid against sc_cw_evaluate on the same wave table and points, and the oracle's
    float64 sum: the factorised form regroups the same sum (FP64 both)."""
    from oracle import scattervolume as osv
    smp = samples.sphere_volume(4, nxy=24, nz=5, size=(20.0, 20.0, 8.0))
    p = solver.make_params(**kw)
    sol = solver.solve(ctx, p, torch.from_numpy(smp).cuda())
    origin, step = (1.3, 2.1, -6.5), (1.1, 1.7, 13.0 / (counts[2] - 1))
    grid = solver.field_grid(ctx, p, sol, origin, step, counts).cpu().numpy().reshape(-1, 3)
    pts = _grid_points(origin, step, counts)
    wt = solver.waves(ctx, p, sol)
    direct = solver.evaluate(ctx, wt.E0, wt.k, wt.z_layers, wt.begin, wt.end, torch.from_numpy(pts).cuda())
    direct = direct.cpu().numpy()
    assert np.linalg.norm(grid - direct) / np.linalg.norm(direct) < 1e-12
    okw = dict(kw)
    if "kappa" in okw:
        okw["kappa"] = (okw["kappa"],)
    po = osv.Params(**okw)
    ref = osv.solve(smp, po)
    W = osv.build_waves(ref, po)
    layers = [(W.z[l], W.Pr_E[l], W.Pr_k[l], W.Pt_E[l], W.Pt_k[l]) for l in range(len(W.z))]
    zl, b, e, WE, Wk = ocw.unpack(W.Pi_E, W.Pi_k, layers)
    if po.external:
        zl = np.array([z if (l == 0 or l == len(zl) - 1) else 0.0 for l, z in enumerate(zl)])
    E_ref = ocw.evaluate(pts, zl, b, e, WE, Wk)
    assert np.linalg.norm(grid - E_ref) / np.linalg.norm(E_ref) < 1e-9
    # complex64 output: the same values rounded
    g32 = solver.field_grid(ctx, p, sol, origin, step, counts, precision=1).cpu().numpy().reshape(-1, 3)
    assert np.linalg.norm(g32 - grid) / np.linalg.norm(grid) < 1e-7


def test_field_grid_slabs_equal_the_whole_grid(ctx):
    """The z-plane split on one GPU, without collectives: the grid evaluated in three slabs (each from its first
    plane, as three ranks would), from a solution copied into empty_solution's buffers (as a rank receives it),
    equals the whole grid; split_field_grid without a process group is field_grid."""
    from scattersim_b200 import fieldsplit
    smp = samples.sphere_volume(4, nxy=24, nz=5, size=(20.0, 20.0, 8.0))
    p = solver.make_params(lambda_=0.6, size=(20, 20, 8), coef=(7, 5), direction=(0.17, 0.05, 0.98), ex=(1, 0),
                           ey=(0, 0))
    sol = solver.solve(ctx, p, torch.from_numpy(smp).cuda())
    origin, step, counts = (1.3, 2.1, -6.5), (1.1, 1.7, 0.55), (9, 7, 23)
    whole = solver.field_grid(ctx, p, sol, origin, step, counts)
    scale = whole.abs().max()
    assert (solver.split_field_grid(ctx, p, sol, origin, step, counts) - whole).abs().max() <= 1e-14 * scale
    recv = solver.empty_solution(ctx, p, smp.shape)
    for dst, src in ((recv.x, sol.x), (recv.evl, sol.evl), (recv.Qc, sol.Qc), (recv.Qh, sol.Qh)):
        assert dst.shape == src.shape
        dst.copy_(src)

    def slab(b, e):
        return solver.field_grid(ctx, p, recv, (origin[0], origin[1], origin[2] + b * step[2]), step,
                                 (counts[0], counts[1], e - b))
    got = fieldsplit.slab_grid(slab, counts, fieldsplit.plane_blocks(counts[2], 3))
    assert got.shape == whole.shape
    assert (got - whole).abs().max() <= 1e-12 * scale
