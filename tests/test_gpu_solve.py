"""End-to-end parity of the scattervolume solve on the GPU against the CPU oracle.

The bar (FP64 plain path): relative error <= 1e-9 on the R/T amplitude vector
and on the electric field evaluated on a grid from the wave lists of the
coupled-wave structure.  Both quantities are invariant to eigenvector scale
and to the labelling of forward/backward modes, which is where the GPU path
and LAPACK legitimately differ.
"""
import numpy as np
import pytest
import torch

from oracle import cw as ocw
from oracle import scattervolume as osv
from scattersim_b200 import samples, solver

pytestmark = pytest.mark.gpu

TOL = 1e-9


def oracle_tables(sol, p, ez_mode=0):
    W = osv.build_waves(sol, p)
    layers = []
    for l in range(len(W.z)):
        PrE, PtE = W.Pr_E[l], W.Pt_E[l]
        if ez_mode == 1:
            PrE = osv.transverse_ez(PrE, W.Pr_k[l]) if len(PrE) else PrE
            PtE = osv.transverse_ez(PtE, W.Pt_k[l]) if len(PtE) else PtE
        layers.append((W.z[l], PrE, W.Pr_k[l], PtE, W.Pt_k[l]))
    PiE = W.Pi_E if ez_mode == 0 else osv.transverse_ez(W.Pi_E, W.Pi_k)
    return ocw.unpack(PiE, W.Pi_k, layers)


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def self_sensitivity(smp, p, seed=0):
    """Relative change of the oracle's R/T under 1e-15 relative noise on the sample."""
    rng = np.random.default_rng(seed)
    a = osv.solve(smp, p, keep=False).x
    b = osv.solve(smp * (1 + 1e-15 * rng.standard_normal(smp.shape)), p, keep=False).x
    return np.linalg.norm(a - b) / np.linalg.norm(a)


def run_case(ctx, smp, p_kw, grid_axis=1, extent=None, center=None, N=48, plane=None, ez_mode=0, tol=TOL):
    p = osv.Params(**p_kw)
    ref = osv.solve(smp, p)
    cp = solver.make_params(**{("lambda_" if k == "lambda_" else k): v for k, v in p_kw.items()})
    dsmp = torch.from_numpy(np.ascontiguousarray(smp)).cuda()
    sol = solver.solve(ctx, cp, dsmp)
    x = sol.x.cpu().numpy()
    assert rel(x, ref.x) < tol, rel(x, ref.x)
    # fields from both wave tables, evaluated by the same float64 sum
    zl, b, e, WE, Wk = oracle_tables(ref, p, ez_mode)
    wt = solver.waves(ctx, cp, sol, ez_mode=ez_mode)
    assert np.array_equal(wt.begin, b) and np.array_equal(wt.end, e)
    assert np.allclose(wt.z_layers, zl)
    size = p.size
    extent = extent or max(size[0], size[2] * 2.5)
    center = center or (size[0] / 2, size[1] / 2, p.z)
    plane = size[1] / 2 if plane is None else plane
    pts = ocw.slice_points(grid_axis, center, extent, N, plane)
    E_ref = ocw.evaluate(pts, zl, b, e, WE, Wk)
    gE = wt.E0.cpu().numpy()
    gK = wt.k.cpu().numpy()
    E_gpu_tab = ocw.evaluate(pts, wt.z_layers, wt.begin, wt.end, gE, gK)
    assert rel(E_gpu_tab, E_ref) < tol, rel(E_gpu_tab, E_ref)
    # GPU evaluator on the GPU table
    E_dev = solver.evaluate(ctx, wt.E0, wt.k, wt.z_layers, wt.begin, wt.end, torch.from_numpy(pts).cuda())
    assert rel(E_dev.cpu().numpy(), E_ref) < tol
    return ref, sol


@pytest.mark.parametrize("seed,M", [(0, (3, 3)), (1, (5, 5)), (2, (7, 5)), (3, (11, 11))])
def test_thin_volume_triangle(ctx, seed, M):
    smp = samples.triangle_map(seed)
    run_case(ctx, smp, dict(lambda_=0.5, size=(10, 10, 1), coef=M, ex=(1, 0), ey=(0, 0)))


def test_even_by_odd_slice_crop_tables(ctx):
    """An even x odd slice goes through the reference's irregular shift tables.

    The slab and wavelength keep the transfer-matrix chain well conditioned
    (oracle self-sensitivity to 1e-15 input noise ~1e-14), so the 1e-9 bar
    holds; thicker slabs at shorter wavelengths amplify evanescent orders
    exponentially in the reference formulation itself.
    """
    rng = np.random.default_rng(9)
    smp = (1.0 + 0.5 * (rng.uniform(size=(1, 12, 9)) > 0.6)).astype(np.complex128)
    kw = dict(lambda_=1.0, size=(10, 10, 0.3), coef=(5, 7), ex=(1, 0), ey=(0, 0))
    assert self_sensitivity(smp, osv.Params(**kw)) < 1e-12
    run_case(ctx, smp, kw)


def test_thin_volume_oblique_ypol(ctx):
    smp = samples.triangle_map(4)
    run_case(ctx, smp, dict(lambda_=0.55, size=(10, 10, 1), coef=(7, 7), direction=(0.2, 0.1, 1)))


def test_multilayer_volume(ctx):
    smp = samples.sphere_volume(0, nxy=32, nz=6, size=(20.0, 20.0, 8.0))
    run_case(ctx, smp, dict(lambda_=0.6, size=(20, 20, 8), coef=(5, 5),
                            direction=(np.sin(np.radians(10)), 0, np.cos(np.radians(10))), ex=(1, 0), ey=(0, 0)))


def test_external_and_npz(ctx):
    smp = samples.sphere_volume(1, nxy=24, nz=4, size=(20.0, 20.0, 8.0))
    run_case(ctx, smp, dict(lambda_=0.6, size=(20, 20, 8), coef=(3, 3), external=True))
    run_case(ctx, smp, dict(lambda_=0.6, size=(20, 20, 8), coef=(3, 3), npz=True))


def test_cw_semantics_transverse_ez(ctx):
    smp = samples.triangle_map(5)
    run_case(ctx, smp, dict(lambda_=0.5, size=(10, 10, 1), coef=(5, 5)), ez_mode=1)


def test_homogeneous_layers_kat(ctx):
    """The M = 1 stack of data/generate_layer_volume.py against the Fresnel solve."""
    from oracle import scatterlayer as osl
    smp = np.array([1.4 + 0.05j, 1.4 + 0j]).reshape(2, 1, 1)
    ref, sol = run_case(ctx, smp, dict(lambda_=1.0, size=(10, 10, 10), coef=(1, 1)), extent=20.0,
                        center=(0, 0, 0), plane=0.0)
    inc, waves, ri, z = osl.solve()
    x = sol.x.cpu().numpy()
    # reflected (wound to z_0) and transmitted (wound to z_last) amplitudes
    r_gpu = x[0:3] * np.exp(1j * (-2 * osv.PI / 1.0) * (-z[0]))
    t_gpu = x[3:6] * np.exp(1j * (2 * osv.PI / 1.0) * (-z[-1]))
    assert np.allclose(r_gpu, waves[0][1][0], atol=1e-7)
    assert np.allclose(t_gpu, waves[-1][2][0], atol=1e-7)


def test_energy_balance(ctx):
    smp = samples.triangle_map(6)
    cp = solver.make_params(lambda_=0.5, size=(10, 10, 1), coef=(9, 9), ex=(1, 0), ey=(0, 0))
    sol = solver.solve(ctx, cp, torch.from_numpy(smp).cuda(), fields=False)
    p = osv.Params(lambda_=0.5, size=(10, 10, 1), coef=(9, 9), ex=(1, 0), ey=(0, 0))
    d, e, dirv, k, ni, slices, num_pixels, z, M, msgs = osv.setup(smp, p)
    lat = osv.upwq_cal(M, p.size, dirv, k, ni)
    MF = M[0] * M[1]
    Sz0 = lat.Sz[0].ravel(order="F")
    Sz1 = lat.Sz[1].ravel(order="F")
    x = sol.x.cpu().numpy()
    R = (np.abs(x[0:3 * MF].reshape(3, MF)) ** 2).sum(0) @ Sz0.real
    T = (np.abs(x[3 * MF:].reshape(3, MF)) ** 2).sum(0) @ Sz1.real
    assert abs(R + T - 1.0) < 1e-10


def test_mixed_precision_solve_matches_oracle(ctx):
    """Transfer-chain, boundary and Pz products on the int8 tensor cores (7 digit
    slices, forced): R/T and fields within 1e-8 of the FP64 oracle."""
    from scattersim_b200 import _lib
    smp = samples.sphere_volume(2, nxy=32, nz=6, size=(20.0, 20.0, 8.0))
    kw = dict(lambda_=0.6, size=(20, 20, 8), coef=(7, 7),
              direction=(np.sin(np.radians(10)), 0, np.cos(np.radians(10))), ex=(1, 0), ey=(0, 0))
    ctx.set_precision(_lib.SC_SWEEP_SLICES(7))
    try:
        run_case(ctx, smp, kw, tol=1e-8)
    finally:
        ctx.set_precision(_lib.SC_SWEEP_FP64)


def test_layer_split_blocks_on_one_gpu(ctx):
    """sc_volume_chain_block on two layer blocks, their ordered product and sc_volume_boundary_solve: the same
    R/T as the unsplit solve and the oracle (the exchange itself is covered by the gloo test)."""
    smp = samples.sphere_volume(3, nxy=32, nz=6, size=(20.0, 20.0, 8.0))
    kw = dict(lambda_=0.6, size=(20, 20, 8), coef=(7, 7),
              direction=(np.sin(np.radians(10)), 0, np.cos(np.radians(10))), ex=(1, 0), ey=(0, 0), external=True)
    p = solver.make_params(**kw)
    d = torch.from_numpy(smp).cuda()
    full = solver.solve(ctx, p, d, fields=False).x.cpu().numpy()
    ref = osv.solve(smp, osv.Params(**kw), keep=False).x
    for cut in (1, 3, 5):
        P0, G0 = solver.chain_block(ctx, p, d, 0, cut)
        P1, G1 = solver.chain_block(ctx, p, d, cut, 6)
        assert G1 is None
        x = solver.boundary_solve(ctx, p, smp.shape, solver.colmajor_matmul(ctx, P1, P0), G0).cpu().numpy()
        assert rel(x, full) < 1e-11
        assert rel(x, ref) < TOL
    # a single block is the whole chain
    P, G = solver.chain_block(ctx, p, d, 0, 6)
    assert rel(solver.boundary_solve(ctx, p, smp.shape, P, G).cpu().numpy(), full) < 1e-12
