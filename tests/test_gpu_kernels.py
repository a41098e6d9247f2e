"""Kernel-level parity on the GPU: GEMM, LU solve, eigensolver, Fourier coefficients, Phi.

Each CUDA kernel is checked against the CPU oracle (numpy/scipy LAPACK stands
in for MKL) on seeded inputs.  Tolerances are relative, FP64.
"""
import numpy as np
import pytest
import torch

from oracle import scattervolume as osv
from scattersim_b200 import samples

pytestmark = pytest.mark.gpu

RNG = np.random.default_rng(1234)


def crand(*shape, rng=RNG):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


def to_dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def colmajor(a):
    """numpy (..., m, n) -> device buffer holding the column-major storage."""
    return to_dev(np.ascontiguousarray(np.swapaxes(a, -1, -2)))


def from_colmajor(t, m, n):
    return np.swapaxes(t.cpu().numpy().reshape(-1, n, m), -1, -2)


@pytest.mark.parametrize("m,n,k,batch", [(1, 1, 1, 1), (7, 5, 3, 2), (64, 64, 16, 1), (130, 67, 95, 3),
                                         (200, 1, 200, 2)])
def test_zgemm(ctx, m, n, k, batch):
    import ctypes
    A, B, C = crand(batch, m, k), crand(batch, k, n), crand(batch, m, n)
    alpha, beta = 0.7 - 0.2j, -1.1 + 0.4j
    dA, dB, dC = colmajor(A), colmajor(B), colmajor(C)
    al = (ctypes.c_double * 2)(alpha.real, alpha.imag)
    be = (ctypes.c_double * 2)(beta.real, beta.imag)
    from scattersim_b200._lib import check
    check(ctx.lib.sc_zgemm_batched(ctx.handle, m, n, k, al, ctypes.c_void_p(dA.data_ptr()), m, m * k,
                                   ctypes.c_void_p(dB.data_ptr()), k, k * n, be, ctypes.c_void_p(dC.data_ptr()), m,
                                   m * n, batch, None))
    torch.cuda.synchronize()
    ref = alpha * A @ B + beta * C
    got = from_colmajor(dC, m, n)
    assert np.abs(got - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max()) * k


@pytest.mark.parametrize("n,nrhs,batch", [(1, 1, 1), (5, 2, 3), (33, 7, 2), (100, 100, 1), (257, 3, 2)])
def test_linearsolve(ctx, n, nrhs, batch):
    import ctypes
    A, B = crand(batch, n, n), crand(batch, n, nrhs)
    dA, dB = colmajor(A), colmajor(B)
    info = (ctypes.c_int * batch)()
    from scattersim_b200._lib import check
    check(ctx.lib.sc_linearsolve_batched(ctx.handle, ctypes.c_void_p(dA.data_ptr()), n,
                                         ctypes.c_void_p(dB.data_ptr()), nrhs, batch, info, None))
    X = from_colmajor(dB, n, nrhs)
    ref = np.linalg.solve(A, B)
    assert np.abs(X - ref).max() / np.abs(ref).max() < 1e-10


def test_linearsolve_singular(ctx):
    import ctypes
    from scattersim_b200._lib import ScatterError, check, SC_SINGULAR
    A = np.zeros((1, 4, 4), complex)
    A[0, 0, 0] = 1
    dA, dB = colmajor(A), colmajor(crand(1, 4, 1))
    info = (ctypes.c_int * 1)()
    with pytest.raises(ScatterError) as e:
        check(ctx.lib.sc_linearsolve_batched(ctx.handle, ctypes.c_void_p(dA.data_ptr()), 4,
                                             ctypes.c_void_p(dB.data_ptr()), 1, 1, info, None))
    assert e.value.status == SC_SINGULAR
    assert info[0] == 2


def _eig_check(A, w, V):
    n = A.shape[-1]
    for b in range(A.shape[0]):
        res = np.linalg.norm(A[b] @ V[b] - V[b] * w[b][None, :]) / (np.linalg.norm(A[b]) * np.sqrt(n))
        assert res < 1e-12, res
        assert np.allclose(np.linalg.norm(V[b], axis=0), 1.0, atol=1e-12)
        ref = np.linalg.eigvals(A[b])
        # multiset match
        d = np.abs(w[b][:, None] - ref[None, :])
        assert d.min(axis=1).max() < 1e-9 * max(1.0, np.abs(ref).max())


@pytest.mark.parametrize("n,batch", [(1, 1), (2, 2), (3, 1), (17, 3), (64, 2), (65, 2), (130, 2), (300, 1)])
def test_eigensolve_random(ctx, n, batch):
    from scattersim_b200.solver import eigensolve
    A = crand(batch, n, n)
    w, V = eigensolve(ctx, to_dev(A))
    _eig_check(A, w.cpu().numpy(), V.cpu().numpy())


def test_eigensolve_degenerate(ctx):
    """Diagonalisable matrices with repeated eigenvalues (homogeneous layers)."""
    from scattersim_b200.solver import eigensolve
    rng = np.random.default_rng(7)
    n = 40
    lam = np.repeat(crand(n // 2, rng=rng), 2)
    Q, _ = np.linalg.qr(crand(n, n, rng=rng))
    A = (Q * lam[None, :]) @ Q.conj().T
    w, V = eigensolve(ctx, to_dev(A[None]))
    w, V = w.cpu().numpy(), V.cpu().numpy()
    _eig_check(A[None], w, V)
    assert np.linalg.cond(V[0]) < 1e6
    D = np.diag(np.full(6, 1.96 + 0j))
    w, V = eigensolve(ctx, to_dev(D[None]))
    assert np.allclose(w.cpu().numpy(), 1.96)
    assert np.linalg.cond(V.cpu().numpy()[0]) < 10


def test_eigensolve_phi_layer(ctx):
    """The 4M x 4M layer matrix of the thin-volume workload at 5x5 orders."""
    from scattersim_b200.solver import eigensolve
    smp = samples.triangle_map(3)
    p = osv.Params(lambda_=0.5, size=(10, 10, 1), coef=(5, 5), ex=(1, 0), ey=(0, 0))
    d, e, dirv, k, ni, slices, num_pixels, z, M, msgs = osv.setup(smp, p)
    lat = osv.upwq_cal(M, p.size, dirv, k, ni)
    P, _, _ = osv.phi(slices[0], M, lat, k)
    w, V = eigensolve(ctx, to_dev(P[None]))
    _eig_check(P[None], w.cpu().numpy(), V.cpu().numpy())


@pytest.mark.parametrize("shape,M", [((1, 64, 64), (11, 11)), ((3, 20, 16), (5, 7)), ((2, 15, 15), (15, 15)),
                                     ((1, 9, 12), (4, 6)), ((2, 10, 7), (5, 7)), ((1, 12, 9), (6, 5))])
def test_fft2_crop(ctx, shape, M):
    import ctypes
    from scattersim_b200._lib import check
    rng = np.random.default_rng(5)
    smp = rng.uniform(1.0, 1.6, shape) + 1j * rng.uniform(0, 0.05, shape)
    slices, _ = osv.reformat(smp)
    Mx, My = M
    Z, S1, S2 = shape
    dS = to_dev(smp)
    Nf = torch.empty(Z * Mx * My, dtype=torch.complex128, device="cuda")
    Nif = torch.empty_like(Nf)
    check(ctx.lib.sc_fft2_crop(ctx.handle, ctypes.c_void_p(dS.data_ptr()), Z, S1, S2, Mx, My,
                               ctypes.c_void_p(Nf.data_ptr()), ctypes.c_void_p(Nif.data_ptr()), None))
    torch.cuda.synchronize()
    got_f = Nf.cpu().numpy().reshape(Z, Mx, My).transpose(0, 2, 1)
    got_i = Nif.cpu().numpy().reshape(Z, Mx, My).transpose(0, 2, 1)
    for z in range(Z):
        ref_f = osv.fftw_fft2(slices[z] ** 2, My, Mx)
        ref_i = osv.fftw_fft2((1 / slices[z]) ** 2, My, Mx)
        assert np.abs(got_f[z] - ref_f).max() < 1e-13 * np.abs(ref_f).max()
        assert np.abs(got_i[z] - ref_i).max() < 1e-13 * np.abs(ref_i).max()


@pytest.mark.parametrize("M,direction", [((5, 5), (0, 0, 1)), ((3, 7), (0.3, -0.2, 1))])
def test_phi(ctx, M, direction):
    import ctypes
    from scattersim_b200._lib import check
    smp = samples.triangle_map(11, n=32)
    p = osv.Params(lambda_=0.6, size=(10, 10, 1), coef=M, direction=direction)
    d, e, dirv, k, ni, slices, num_pixels, z, Mc, msgs = osv.setup(smp, p)
    lat = osv.upwq_cal(Mc, p.size, dirv, k, ni)
    P, Nf, Nif = osv.phi(slices[0], Mc, lat, k)
    Mx, My = Mc
    dNf = to_dev(Nf.T.copy())
    dNif = to_dev(Nif.T.copy())
    n = 4 * Mx * My
    dP = torch.empty(n * n, dtype=torch.complex128, device="cuda")
    up = (ctypes.c_double * Mx)(*lat.up)
    wq = (ctypes.c_double * My)(*lat.wq)
    check(ctx.lib.sc_phi(ctx.handle, ctypes.c_void_p(dNf.data_ptr()), ctypes.c_void_p(dNif.data_ptr()), 1, Mx, My,
                         up, wq, k, ctypes.c_void_p(dP.data_ptr()), None))
    got = dP.cpu().numpy().reshape(n, n).T
    assert np.abs(got - P).max() <= 1e-14 * np.abs(P).max()
