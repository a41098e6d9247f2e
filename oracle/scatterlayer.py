"""Oracle: closed-form homogeneous multilayer solve of scatterlayer (test infrastructure only).

Restates ``ScatterLayer.cpp:110-266`` for ONE incident plane wave (``--alpha 0``).
It is the known-answer cross-check the reference implies in
``data/generate_layer_volume.py:1-2``: scattervolume on a stack of homogeneous
slices at one Fourier order must reproduce it.
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sla

from .scattervolume import orthogonalize


def idx(layer, d, c):
    """ScatterLayer.cpp:77-79 (d: 0 = transmitted, 1 = reflected)."""
    return layer * 6 + d * 3 + c


def solve(lambda_=1.0, direction=(0, 0, 1), ex=(0, 0), ey=(1, 0), ez=(0, 0),
          n=(1, 1.4, 1.4, 1.0), kappa=(0.05,), z=(-5.0, 0.0, 5.0)):
    """ScatterLayer.cpp:281-420 for a single plane wave.

    Returns (waves, ri, z) where waves = list over boundaries l of
    (z_l, (r_E, r_k), (t_E, t_k)), each wave already wound by -z_l like the
    ``.cw`` writer (:404-409).
    """
    n, kappa, z = list(n), list(kappa), list(z)
    L = max(len(n), len(kappa) + 1, len(z) + 1)                 # :329-333
    n += [n[-1]] * (L - len(n))                                  # :337
    kappa += [0.0] * (L - 1 - len(kappa))                        # :338
    while len(z) + 1 < L:                                        # :339-343
        z.append(z[-1] + 10.0)
    d = np.array(direction, dtype=np.float64)
    d = d / np.linalg.norm(d)
    e = orthogonalize(np.array([complex(*ex), complex(*ey), complex(*ez)]), d)
    d = d * n[0]
    k_vac = 2 * np.pi / lambda_                                  # :351 (M_PI)
    k = k_vac
    ri = [complex(n[0], 0.0)] + [complex(n[l], kappa[l - 1]) for l in range(1, L)]
    # tira::planewave::getDirection() of i_ref = unit real k; s = dir * n0  (:133)
    s = d / np.linalg.norm(d) * n[0]
    sz = [np.sqrt(ri[l] * ri[l] - s[0] * s[0] - s[1] * s[1]) for l in range(L)]
    A = np.zeros((6 * L, 6 * L), dtype=np.complex128)
    b = np.zeros(6 * L, dtype=np.complex128)
    T, R = 0, 1
    # SetBoundaryConditions (:152-165)
    for c in range(3):
        A[c, idx(0, T, c)] = 1
        b[c] = e[c]
        A[3 + c, idx(L - 1, R, c)] = 1
    # SetGaussianConstraints (:167-184)
    row = 6
    for l in range(L - 1):
        A[row + l, idx(l, R, 0)] = s[0]
        A[row + l, idx(l, R, 1)] = s[1]
        A[row + l, idx(l, R, 2)] = -sz[l]
    row += L - 2
    for l in range(1, L):
        A[row + l, idx(l, T, 0)] = s[0]
        A[row + l, idx(l, T, 1)] = s[1]
        A[row + l, idx(l, T, 2)] = sz[l]
    # SetBoundaryConstraints (:186-232)
    row = 6 + 2 * (L - 1)
    X, Y, Zc = 0, 1, 2
    for l in range(L - 1):
        zn = z[l] if l == 0 else z[l] - z[l - 1]
        zp = 0.0 if l == L - 2 else z[l] - z[l + 1]
        et = np.exp(1j * k * sz[l] * zn)
        er = np.exp(-1j * k * sz[l + 1] * zp)
        r0 = row + 4 * l
        A[r0, idx(l, T, X)] = et
        A[r0, idx(l, R, X)] = 1.0
        A[r0, idx(l + 1, T, X)] = -1.0
        A[r0, idx(l + 1, R, X)] = -er
        A[r0 + 1, idx(l, T, Y)] = et
        A[r0 + 1, idx(l, R, Y)] = 1.0
        A[r0 + 1, idx(l + 1, T, Y)] = -1.0
        A[r0 + 1, idx(l + 1, R, Y)] = -er
        A[r0 + 2, idx(l, T, Zc)] = s[1] * et
        A[r0 + 2, idx(l, T, Y)] = -sz[l] * et
        A[r0 + 2, idx(l, R, Zc)] = s[1]
        A[r0 + 2, idx(l, R, Y)] = sz[l]
        A[r0 + 2, idx(l + 1, T, Zc)] = -s[1]
        A[r0 + 2, idx(l + 1, T, Y)] = sz[l + 1]
        A[r0 + 2, idx(l + 1, R, Zc)] = -s[1] * er
        A[r0 + 2, idx(l + 1, R, Y)] = -sz[l + 1] * er
        A[r0 + 3, idx(l, T, X)] = sz[l] * et
        A[r0 + 3, idx(l, T, Zc)] = -s[0] * et
        A[r0 + 3, idx(l, R, X)] = -sz[l]
        A[r0 + 3, idx(l, R, Zc)] = -s[0]
        A[r0 + 3, idx(l + 1, T, X)] = -sz[l + 1]
        A[r0 + 3, idx(l + 1, T, Zc)] = s[0]
        A[r0 + 3, idx(l + 1, R, X)] = sz[l + 1] * er
        A[r0 + 3, idx(l + 1, R, Zc)] = s[0] * er
    x = sla.solve(A, b)                                          # :399
    waves = []
    for l in range(L - 1):                                       # mat2waves :240-266
        rk = np.array([s[0] * k_vac, s[1] * k_vac, -sz[l] * k_vac])
        tk = np.array([s[0] * k_vac, s[1] * k_vac, sz[l + 1] * k_vac])
        rE = x[[idx(l, R, 0), idx(l, R, 1), idx(l, R, 2)]]
        tE = x[[idx(l + 1, T, 0), idx(l + 1, T, 1), idx(l + 1, T, 2)]]
        rE = rE * np.exp(1j * rk[2] * (-z[l]))                  # wind(0,0,-z_l)
        tE = tE * np.exp(1j * tk[2] * (-z[l]))
        waves.append((z[l], (rE, rk), (tE, tk)))
    inc = (np.asarray(e), np.array([d[0] * k, d[1] * k, d[2] * k]))
    return inc, waves, ri, z
