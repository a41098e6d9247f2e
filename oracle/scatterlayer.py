"""Oracle: homogeneous multilayer and single-interface solves (test infrastructure only).

Restates, per incident plane wave,

* ``ScatterLayer.cpp:110-266`` -- the 6L x 6L system of one plane wave in a
  stack of L homogeneous layers (boundary conditions, Gaussian constraints,
  tangential E/H continuity), its solve, and ``mat2waves``;
* the layer bookkeeping of ``ScatterLayer.cpp:321-343`` (L from the longest
  option list, padding of n, kappa and z);
* tira's ``planewave::SolidAnglePolar`` focused-beam sampling as the shipped
  files pin it (``beam_polar``): ``data/psf.cw`` and ``x64/a.cw`` carry the
  beams of scatterplane's and scatterlayer's default runs;
* scatterplane's one-interface solve (``ScatterPlane.cpp:81-264``) as the
  L = 2 case of the layer system.

The known answers: scattervolume on a homogeneous stack at one Fourier order
equals ``solve`` (data/generate_layer_volume.py:1-2); every record of
data/psf.cw and every incident and transmitted record of x64/a.cw is
reproduced from the restated beams (with the record frame of
``oracle.cw.get_e0_tira``).
"""
from __future__ import annotations

import numpy as np
import scipy.linalg as sla

from .cw import tira_frame
from .scattervolume import orthogonalize

T, R = 0, 1          # ScatterLayer.cpp:73-75 (Transmitted, Reflected)


def idx(layer, d, c):
    """ScatterLayer.cpp:77-79: unknown index of (layer, direction, coordinate)."""
    return layer * 6 + d * 3 + c


def fill_layers(n, kappa, z):
    """ScatterLayer.cpp:321-343: L = the longest of n, kappa + 1, z + 1; pad the others."""
    n, kappa, z = [float(v) for v in n], [float(v) for v in kappa], [float(v) for v in z]
    L = max(len(n), len(kappa) + 1, len(z) + 1)
    n += [n[-1]] * (L - len(n))
    kappa += [0.0] * (L - 1 - len(kappa))
    kappa = kappa[:L - 1]
    while len(z) + 1 < L:
        z.append(z[-1] + 10.0)
    ri = [complex(n[0], 0.0)] + [complex(n[l], kappa[l - 1]) for l in range(1, L)]   # :116-118
    return L, n, kappa, z[:L - 1], ri


def system(k_in, E0, ri, z, k_vac, n0):
    """ScatterLayer.cpp:133-232: the matrix A and right-hand side b of one incident wave.

    k_in: the incident wave vector (its real direction is used), E0: its
    Cartesian E0.  sz uses the direction scaled by n0 (InitSz :133-148); the
    Gaussian and continuity rows use the unit direction (:167-232).
    """
    L = len(ri)
    d = np.real(np.asarray(k_in, dtype=np.complex128))
    d = d / np.linalg.norm(d)                                   # getDirection()
    s = d * n0
    sz = [np.sqrt(r * r - s[0] * s[0] - s[1] * s[1]) for r in ri]
    A = np.zeros((6 * L, 6 * L), dtype=np.complex128)
    b = np.zeros(6 * L, dtype=np.complex128)
    for c in range(3):                                          # SetBoundaryConditions :152-165
        A[c, idx(0, T, c)] = 1.0
        b[c] = E0[c]
        A[3 + c, idx(L - 1, R, c)] = 1.0
    row = 6                                                     # SetGaussianConstraints :167-184
    for l in range(L - 1):
        A[row + l, idx(l, R, 0)] = d[0]
        A[row + l, idx(l, R, 1)] = d[1]
        A[row + l, idx(l, R, 2)] = -sz[l]
    row += L - 2
    for l in range(1, L):
        A[row + l, idx(l, T, 0)] = d[0]
        A[row + l, idx(l, T, 1)] = d[1]
        A[row + l, idx(l, T, 2)] = sz[l]
    row = 6 + 2 * (L - 1)                                       # SetBoundaryConstraints :186-232
    X, Y, Z = 0, 1, 2
    for l in range(L - 1):
        zn = z[l] if l == 0 else z[l] - z[l - 1]
        zp = 0.0 if l == L - 2 else z[l] - z[l + 1]
        et = np.exp(1j * k_vac * sz[l] * zn)
        er = np.exp(-1j * k_vac * sz[l + 1] * zp)
        r0 = row + 4 * l
        A[r0, idx(l, T, X)] = et
        A[r0, idx(l, R, X)] = 1.0
        A[r0, idx(l + 1, T, X)] = -1.0
        A[r0, idx(l + 1, R, X)] = -er
        A[r0 + 1, idx(l, T, Y)] = et
        A[r0 + 1, idx(l, R, Y)] = 1.0
        A[r0 + 1, idx(l + 1, T, Y)] = -1.0
        A[r0 + 1, idx(l + 1, R, Y)] = -er
        A[r0 + 2, idx(l, T, Z)] = d[1] * et
        A[r0 + 2, idx(l, T, Y)] = -sz[l] * et
        A[r0 + 2, idx(l, R, Z)] = d[1]
        A[r0 + 2, idx(l, R, Y)] = sz[l]
        A[r0 + 2, idx(l + 1, T, Z)] = -d[1]
        A[r0 + 2, idx(l + 1, T, Y)] = sz[l + 1]
        A[r0 + 2, idx(l + 1, R, Z)] = -d[1] * er
        A[r0 + 2, idx(l + 1, R, Y)] = -sz[l + 1] * er
        A[r0 + 3, idx(l, T, X)] = sz[l] * et
        A[r0 + 3, idx(l, T, Z)] = -d[0] * et
        A[r0 + 3, idx(l, R, X)] = -sz[l]
        A[r0 + 3, idx(l, R, Z)] = -d[0]
        A[r0 + 3, idx(l + 1, T, X)] = -sz[l + 1]
        A[r0 + 3, idx(l + 1, T, Z)] = d[0]
        A[r0 + 3, idx(l + 1, R, X)] = sz[l + 1] * er
        A[r0 + 3, idx(l + 1, R, Z)] = d[0] * er
    return A, b, s, sz


def solve_wave(k_in, E0, ri, z, k_vac, n0):
    """One incident wave through the stack (ScatterLayer.cpp:389-410).

    Returns [(z_l, r_E, r_k, t_E, t_k)] per boundary l, each wave wound by -z_l
    as the .cw writer stores it (:404-409).  The reference solves with
    colPivHouseholderQr; any backward-stable solve of the same square system
    agrees to rounding.
    """
    A, b, s, sz = system(k_in, E0, ri, z, k_vac, n0)
    x = sla.solve(A, b)
    out = []
    for l in range(len(ri) - 1):                                # mat2waves :240-266
        rk = np.array([s[0] * k_vac, s[1] * k_vac, -sz[l] * k_vac])
        tk = np.array([s[0] * k_vac, s[1] * k_vac, sz[l + 1] * k_vac])
        rE = x[[idx(l, R, 0), idx(l, R, 1), idx(l, R, 2)]] * np.exp(-1j * rk[2] * z[l])
        tE = x[[idx(l + 1, T, 0), idx(l + 1, T, 1), idx(l + 1, T, 2)]] * np.exp(-1j * tk[2] * z[l])
        out.append((z[l], rE, rk, tE, tk))
    return out


def beam_polar(alpha, k_center, e_center, N0, N1, beta=0.0):
    """tira::planewave::SolidAnglePolar as the shipped files pin it.

    Wave t = j * N0 + i (theta inner, phi outer), theta_i = beta + i dtheta,
    dtheta = (alpha - beta) / N0, phi_j = j 2 pi / N1.  Its direction is
    R_c (sin th cos ph, sin th sin ph, cos th), R_c = tira_frame(k_center), and
    its record pair is the centre wave's pair scaled by sin(theta) dtheta dphi
    (so E0 = w R_t (a, b, 0) with (a, b, 0) = R_c^T e_center).  Pinned for
    beta = 0 by data/psf.cw (alpha 0.5 about (1, 0, 1)) and x64/a.cw (alpha 1
    about z); beta > 0 is unpinned.  Returns (k (N, 3) real, E0 (N, 3) complex).
    """
    kc = np.asarray(k_center, dtype=np.float64)
    kmag = np.linalg.norm(kc)
    Rc = tira_frame(kc)
    loc = Rc.T @ np.asarray(e_center, dtype=np.complex128)
    loc[2] = 0.0
    dth = (alpha - beta) / N0
    dph = 2.0 * np.pi / N1
    ks = np.zeros((N0 * N1, 3))
    Es = np.zeros((N0 * N1, 3), dtype=np.complex128)
    for j in range(N1):
        ph = j * dph
        for i in range(N0):
            th = beta + i * dth
            kh = Rc @ np.array([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)])
            t = j * N0 + i
            ks[t] = kmag * kh
            Es[t] = np.sin(th) * dth * dph * (tira_frame(ks[t]) @ loc)
    return ks, Es


def incident(lambda_, direction, ex, ey, ez, n0):
    """ScatterLayer.cpp:345-353 / ScatterPlane.cpp:136-142: k vector and E0 of the centre wave."""
    d = np.asarray(direction, dtype=np.float64)
    d = d / np.linalg.norm(d)
    e = orthogonalize(np.array([complex(*ex), complex(*ey), complex(*ez)]), d)
    return d * n0 * (2 * np.pi / lambda_), e


def scatterlayer(lambda_=1.0, direction=(0, 0, 1), ex=(0, 0), ey=(1, 0), ez=(0, 0),
                 n=(1, 1.4, 1.4, 1.0), kappa=(0.05,), z=(-5.0, 0.0, 5.0), alpha=1.0, beta=0.0,
                 samples=(64, 64)):
    """ScatterLayer.cpp:281-420 (polar mode).  Returns (Pi_k, Pi_E, layers) in Cartesian E."""
    L, n, kappa, z, ri = fill_layers(n, kappa, z)
    k_vac = 2 * np.pi / lambda_
    kc, e = incident(lambda_, direction, ex, ey, ez, n[0])
    N0, N1 = samples if len(samples) == 2 else (int(np.sqrt(samples[0])),) * 2
    if alpha == 0 or N0 * N1 == 1:
        ks, Es = kc[None, :], e[None, :]
    else:
        ks, Es = beam_polar(alpha, kc, e, N0, N1, beta)
    per = [solve_wave(ks[t], Es[t], ri, z, k_vac, n[0]) for t in range(len(ks))]
    layers = []
    for l in range(L - 1):
        layers.append((z[l], np.array([p[l][1] for p in per]), np.array([p[l][2] for p in per]),
                       np.array([p[l][3] for p in per]), np.array([p[l][4] for p in per])))
    return ks.astype(np.complex128), Es, layers


def scatterplane(lambda_=1.0, direction=(1, 0, 1), focus=(0, 0, 0), ex=(0, 0), ey=(1, 0), ez=(0, 0),
                 n=(1.0, 1.4), kappa=0.05, z=0.0, alpha=0.5, beta=0.0, samples=(64, 64)):
    """ScatterPlane.cpp:81-264 (polar mode) as the L = 2 layer solve.

    Every wave is wound to the focal point (E0 exp(-i k . f)) before the
    interface solve.  Returns (Pi_k, Pi_E, [(z, Pr_E, Pr_k, Pt_E, Pt_k)]).
    """
    ri = [complex(n[0], 0.0), complex(n[1], kappa)]
    k_vac = 2 * np.pi / lambda_
    kc, e = incident(lambda_, direction, ex, ey, ez, n[0])
    N0, N1 = samples if len(samples) == 2 else (int(np.sqrt(samples[0])),) * 2
    if alpha == 0 or N0 * N1 == 1:
        ks, Es = kc[None, :], e[None, :]
    else:
        ks, Es = beam_polar(alpha, kc, e, N0, N1, beta)
    f = np.asarray(focus, dtype=np.float64)
    Es = Es * np.exp(-1j * (ks @ f))[:, None]
    per = [solve_wave(ks[t], Es[t], ri, [z], k_vac, n[0])[0] for t in range(len(ks))]
    layer = (z, np.array([p[1] for p in per]), np.array([p[2] for p in per]),
             np.array([p[3] for p in per]), np.array([p[4] for p in per]))
    return ks.astype(np.complex128), Es, [layer]


def solve(lambda_=1.0, direction=(0, 0, 1), ex=(0, 0), ey=(1, 0), ez=(0, 0),
          n=(1, 1.4, 1.4, 1.0), kappa=(0.05,), z=(-5.0, 0.0, 5.0)):
    """ScatterLayer.cpp:281-420 for the single centre wave (--alpha 0).

    Returns (inc, waves, ri, z) with waves = [(z_l, (r_E, r_k), (t_E, t_k))].
    """
    L, n, kappa, z, ri = fill_layers(n, kappa, z)
    kc, e = incident(lambda_, direction, ex, ey, ez, n[0])
    per = solve_wave(kc, e, ri, z, 2 * np.pi / lambda_, n[0])
    waves = [(zl, (rE, rk), (tE, tk)) for (zl, rE, rk, tE, tk) in per]
    return (np.asarray(e), kc), waves, ri, z
