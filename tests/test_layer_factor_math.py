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


def _factored(B, C, kdz):
    Om = B @ C
    s = _scalings(kdz * kdz * np.abs(Om).sum(0).max())
    h = math.ldexp(kdz, -s)
    y = -(h * h) * Om                                   # (t / 2^s)^2 Omega with t = i kdz
    I = np.eye(len(B))
    Y2, Y3 = y @ y, y @ y @ y
    Y4 = Y2 @ Y2
    out = []
    for which in (0, 1):
        c = [1.0 / math.factorial(2 * j + which) for j in range(13)]
        P1 = c[8] * I + c[9] * y + c[10] * Y2 + c[11] * Y3 + c[12] * Y4
        P2 = c[4] * I + c[5] * y + c[6] * Y2 + c[7] * Y3 + Y4 @ P1
        out.append(c[0] * I + c[1] * y + c[2] * Y2 + c[3] * Y3 + Y4 @ P2)
    F, G = out
    for _ in range(s - 1):                              # double-angle steps to the half angle
        F, G = 2 * F @ F - I, G @ F
    return F, G @ B, C @ G, s


def _apply(F, GB, CG, kdz, X):
    n = len(F)
    t = 1j * kdz
    X1, X2 = X[:n], X[n:]
    U, V = GB @ X2, F @ X1
    P, Q = 2 * V - t * U, (t * t / 2) * U - t * V
    return np.vstack([F @ P - X1, X2 + CG @ Q])


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
