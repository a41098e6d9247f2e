"""The arithmetic of the batched sweep's layer factors, restated in numpy (no GPU).

The sweep replaces the reference's eigen-based layer factor GC_i GD_i^-1 by the
matrix function exp(-t Phi), t = i k dz, Phi = [[0, B], [C, 0]], evaluated as
series in y = (t / 2^s)^2 B C (degree 12, Paterson-Stockmeyer in y^4) with s
double-angle steps chosen per layer, kept at the half angle in factored form
(F, G B, C G) and applied to X = [X1; X2] by four products.  This test runs
exactly that sequence of steps in float64 and compares it with scipy's
expm(-t Phi) X on layers of the workload's kind of norms.
"""
import math

import numpy as np
import pytest
import scipy.linalg as sla


def _scalings(v):
    s = 1
    while s < 60 and v / 4.0 ** s > 4.0:
        s += 1
    return s


def _factored(B, C, kdz, mm=np.matmul):
    Om = mm(B, C)
    s = _scalings(kdz * kdz * np.abs(Om).sum(0).max())
    h = math.ldexp(kdz, -s)
    y = -(h * h) * Om                                   # (t / 2^s)^2 Omega with t = i kdz
    I = np.eye(len(B))
    Y2 = mm(y, y)
    Y3 = mm(Y2, y)
    Y4 = mm(Y2, Y2)
    out = []
    for which in (0, 1):
        c = [1.0 / math.factorial(2 * j + which) for j in range(13)]
        P1 = c[8] * I + c[9] * y + c[10] * Y2 + c[11] * Y3 + c[12] * Y4
        P2 = c[4] * I + c[5] * y + c[6] * Y2 + c[7] * Y3 + mm(Y4, P1)
        out.append(c[0] * I + c[1] * y + c[2] * Y2 + c[3] * Y3 + mm(Y4, P2))
    F, G = out
    for _ in range(s - 1):                              # double-angle steps to the half angle
        F, G = 2 * mm(F, F) - I, mm(G, F)
    return F, mm(G, B), mm(C, G), s


def _apply(F, GB, CG, kdz, X, mm=np.matmul):
    n = len(F)
    t = 1j * kdz
    X1, X2 = X[:n], X[n:]
    U, V = mm(GB, X2), mm(F, X1)
    P, Q = 2 * V - t * U, (t * t / 2) * U - t * V
    return np.vstack([mm(F, P) - X1, X2 + mm(CG, Q)])


@pytest.mark.parametrize("n,scale,kdz", [(6, 0.3, 0.8), (10, 1.0, 3.0), (8, 2.0, 6.0), (12, 0.5, 12.0)])
def test_factored_layer_matches_expm(n, scale, kdz):
    rng = np.random.default_rng(n)
    B = (rng.normal(size=(n, n)) + 1j * rng.normal(size=(n, n))) * scale
    C = (rng.normal(size=(n, n)) + 0.1j * rng.normal(size=(n, n))) * scale
    X = rng.normal(size=(2 * n, 5)) + 1j * rng.normal(size=(2 * n, 5))
    Phi = np.block([[np.zeros((n, n)), B], [C, np.zeros((n, n))]])
    ref = sla.expm(-1j * kdz * Phi) @ X
    F, GB, CG, s = _factored(B, C, kdz)
    got = _apply(F, GB, CG, kdz, X)
    assert s >= 1
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-12


def test_per_layer_scaling_counts():
    # ||y||_1 <= 4 after s steps, and s is the least such count (at least 1)
    for v in [0.1, 3.9, 4.0, 16.1, 64.0, 64.1, 1e6]:
        s = _scalings(v)
        assert v / 4.0 ** s <= 4.0 and (s == 1 or v / 4.0 ** (s - 1) > 4.0)


CRT_MODULI = [255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197]


def _modular_mm(nmod):
    """A B as the modular int8 engine rounds it: rows of A and columns of B scaled by powers of two and rounded
    to al = be = floor((log2 P - 3 - log2 2k) / 2) bits (P the product of the first `nmod` moduli), the
    product of the rounded operands then exact (here FP64, whose error is below the rounding's)."""
    lp = math.log2(math.prod(CRT_MODULI[:nmod]))

    def rows(A, bits):
        m = np.maximum(np.abs(A.real), np.abs(A.imag)).max(axis=1)
        e = np.frexp(np.where(m > 0, m, 1.0))[1]
        sc = np.ldexp(1.0, bits - e)[:, None]
        return (np.round(A.real * sc) + 1j * np.round(A.imag * sc)) / sc

    def mm(A, B):
        bits = min(49, int((lp - 3 - math.log2(2 * A.shape[1])) // 2))
        return rows(A, bits) @ rows(B.T, bits).T
    return mm


def test_modular_rounding_error_scales_with_the_modulus_count():
    """The sweep's layer factors from the oracle's own Phi (a 15x15-order sweep layer pair), every product
    rounded as the modular engine rounds it: 14 moduli (48-bit operands at this depth) stay near FP64, and
    each modulus dropped (about 4 bits) costs about 16x -- the error model for choosing fewer moduli."""
    from oracle import scattervolume as osv
    from scattersim_b200 import samples
    it = samples.sweep_instances(21, count=8, n=64, period=25.0)[3]
    it.orders = 15
    p = osv.Params(**it.params_kw())
    _, _, dirv, k, ni, slices, _, z, M, _ = osv.setup(it.maps, p)
    lat = osv.upwq_cal(M, p.size, dirv, k, ni)
    MF = M[0] * M[1]
    X0 = np.random.default_rng(0).normal(size=(4 * MF, 4)) + 0j
    out = {}
    for nmod in (None, 14, 13, 12):
        mm = np.matmul if nmod is None else _modular_mm(nmod)
        X = X0
        for sl in slices[:2]:
            P, _, _ = osv.phi(sl, M, lat, k)
            F, GB, CG, _ = _factored(P[:2 * MF, 2 * MF:], P[2 * MF:, :2 * MF], k * (z[1] - z[0]), mm)
            X = _apply(F, GB, CG, k * (z[1] - z[0]), X, mm)
        out[nmod] = X
    err = {m: np.linalg.norm(out[m] - out[None]) / np.linalg.norm(out[None]) for m in (14, 13, 12)}
    assert err[14] < 2e-12
    assert 4 < err[13] / err[14] < 64 and 4 < err[12] / err[13] < 64
    assert err[12] < 1e-9
