"""Oracle: literal CPU restatement of scattervolume (test infrastructure only).

Every function follows one piece of the reference and cites it by
file:line.  LAPACK ``zgeev``/``zgesv`` and BLAS ``zgemm`` come from scipy's
bundled OpenBLAS and stand in for Intel MKL (third_Lapack.h:37-85); numpy's
pocketfft stands in for FFTW (same unnormalised forward transform
e^{-2 pi i jk/N}).  The restatement keeps the reference's quirks on purpose:
the transpose on load, the circulant order wrap, the row-major vs
column-major order indexing, the truncated PI macro, the ``kz * n`` factor of
the reflected/transmitted waves and the noise-ordered eigenvalue pairing.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may use this module.
"""
from __future__ import annotations

import functools
import math
from dataclasses import dataclass, field

import numpy as np
import scipy.linalg as sla

PI = 3.141592653            # FourierWave.h:18  (#define PI 3.141592653)
M_PI = math.pi              # math.h M_PI, used at ScatterVolume.cpp:813-814
DBL_EPS = float(np.finfo(np.float64).eps)


# --------------------------------------------------------------------------
# small helpers (FourierWave.h:24-39)
# --------------------------------------------------------------------------
def cross(E, d):
    """FourierWave.h:24-30."""
    return np.array([E[1] * d[2] - E[2] * d[1],
                     E[2] * d[0] - E[0] * d[2],
                     E[0] * d[1] - E[1] * d[0]], dtype=np.complex128)


def orthogonalize(E, d):
    """FourierWave.h:32-39: E /= sqrt(Ex^2+Ey^2+Ez^2) (complex squares), then d x (E x d)."""
    E = np.asarray(E, dtype=np.complex128)
    mag = np.sqrt(E[0] ** 2 + E[1] ** 2 + E[2] ** 2)
    E = E / mag
    dc = np.asarray(d, dtype=np.complex128)
    s = cross(E, dc)
    return cross(dc, s)


# --------------------------------------------------------------------------
# a1/a2: sample load + reformat (FourierWave.h:263-301)
# --------------------------------------------------------------------------
def reformat(data: np.ndarray):
    """FourierWave.h:283-301.

    Each slice is an Eigen column-major Map of shape (shape[1], shape[2]) over
    the C-order .npy buffer, i.e. ``E(r, c) = flat[r + c * shape[1]]``.  For a
    square slice this is the transpose of the .npy slice.  A 2-D array becomes
    one layer.  Returns (slices, shape) with shape = (Z, S1, S2).
    """
    data = np.ascontiguousarray(data, dtype=np.complex128)
    if data.ndim == 2:
        data = data[None]
    if data.ndim != 3:
        raise ValueError("sample must be 2-D or 3-D")
    Z, S1, S2 = data.shape
    flat = data.reshape(-1)
    slices = [flat[i * S1 * S2:(i + 1) * S1 * S2].reshape(S2, S1).T.copy()
              for i in range(Z)]
    return slices, (Z, S1, S2)


# --------------------------------------------------------------------------
# a3: FFT + shift + crop (FourierWave.h:82-195)
# --------------------------------------------------------------------------
def fft_shift2d(mat: np.ndarray) -> np.ndarray:
    """FourierWave.h:82-145 (MATLAB-style fftshift by index tables)."""
    m, n = mat.shape
    if m % 2 == 1:
        p, q = m // 2, n // 2
    else:
        p, q = -(-m // 2), -(-n // 2)
    indx = np.empty(m, dtype=np.int64)
    indy = np.empty(n, dtype=np.int64)
    if m % 2 == 1:
        for i in range(0, m - p - 1):
            indx[i] = (m - p) + i
        for i in range(m - p - 1, m):
            indx[i] = i - (m - p - 1)
    else:
        for i in range(0, m - p):
            indx[i] = p + i
        for i in range(m - p, m):
            indx[i] = i - (m - p)
    if n % 2 == 1:
        for i in range(0, n - q - 1):
            indy[i] = (n - q) + i
        for i in range(n - q - 1, n):
            indy[i] = i - (n - q - 1)
    else:
        for i in range(0, n - q):
            indy[i] = q + i
        for i in range(n - q, n):
            indy[i] = i - (n - q)
    return mat[np.ix_(indx, indy)]


def fftw_fft2(A: np.ndarray, M1: int, M2: int) -> np.ndarray:
    """FourierWave.h:152-195: forward 2-D DFT / (N1 N2), fftshift, centred M1 x M2 crop."""
    N1, N2 = A.shape
    B = np.fft.fft2(A) / N1 / N2
    S = fft_shift2d(B)
    r0, c0 = N1 // 2 - M1 // 2, N2 // 2 - M2 // 2
    return S[r0:r0 + M1, c0:c0 + M2].copy()


# --------------------------------------------------------------------------
# a4/a5: wave-vector lattice + layer matrix (FourierWave.h:319-397)
# --------------------------------------------------------------------------
def lin_spaced(size: int, low: float, high: float) -> np.ndarray:
    """Eigen::VectorXd::setLinSpaced (size 1 yields `high`)."""
    if size == 1:
        return np.array([high], dtype=np.float64)
    step = (high - low) / (size - 1)
    return low + step * np.arange(size, dtype=np.float64)


@dataclass
class Lattice:
    """Output of volume::UpWq_Cal (FourierWave.h:319-334)."""
    p_series: np.ndarray
    q_series: np.ndarray
    up: np.ndarray           # (Mx,)  2 PI p / size_x + dir_x k
    wq: np.ndarray           # (My,)
    Sx: np.ndarray           # up / k
    Sy: np.ndarray
    meshS0: np.ndarray       # (My, Mx)  meshS0[r, c] = Sx[c]
    meshS1: np.ndarray       # (My, Mx)  meshS1[r, c] = Sy[r]
    Sz: list                 # [Sz_top, Sz_bot] (My, Mx)


def upwq_cal(M, size, dirv, k: float, n_layers) -> Lattice:
    """FourierWave.h:319-334 (uses the truncated PI macro)."""
    Mx, My = int(M[0]), int(M[1])
    p_series = lin_spaced(Mx, -float(Mx // 2), float((Mx - 1) // 2))
    q_series = lin_spaced(My, -float(My // 2), float((My - 1) // 2))
    up = 2 * PI * p_series / size[0] + dirv[0] * k * np.ones(Mx)
    wq = 2 * PI * q_series / size[1] + dirv[1] * k * np.ones(My)
    Sx = (up / k).astype(np.complex128)
    Sy = (wq / k).astype(np.complex128)
    meshS0 = np.tile(Sx[None, :], (My, 1))
    meshS1 = np.tile(Sy[:, None], (1, Mx))
    n0, n1 = complex(n_layers[0]), complex(n_layers[1])
    Sz0 = np.sqrt(n0 ** 2 * np.ones((My, Mx)) - meshS0 ** 2 - meshS1 ** 2)
    Sz1 = np.sqrt(n1 ** 2 * np.ones((My, Mx)) - meshS0 ** 2 - meshS1 ** 2)
    return Lattice(p_series, q_series, up, wq, Sx, Sy, meshS0, meshS1, [Sz0, Sz1])


def conv_index(Mx: int, My: int):
    """Circulant coefficient lookup of FourierWave.h:366-372.

    Returns (rowidx, colidx) arrays of shape (M, M) such that the convolution
    entry for Phi row r = qi*Mx+pi and column j = qj*Mx+pj is
    ``N[rowidx[r, j], colidx[r, j]]``.
    """
    MF = Mx * My
    r = np.arange(MF)
    qi, pi_ = r // Mx, r % Mx
    # (int)q % M in C++ keeps the sign, and |q| < M, so it is q itself.
    qs = (np.arange(My) - My // 2)
    ps = (np.arange(Mx) - Mx // 2)
    indR = (qs[qi][:, None] - qs[qi][None, :] + My) % My
    indC = (ps[pi_][:, None] - ps[pi_][None, :] + Mx) % Mx
    return (indR + My // 2) % My, (indC + Mx // 2) % Mx


def phi(sample: np.ndarray, M, lat: Lattice, k: float):
    """volume::phi (FourierWave.h:336-397).  Returns (Phi, Nf, Nif)."""
    Mx, My = int(M[0]), int(M[1])
    Nf = fftw_fft2(sample ** 2, My, Mx)                       # :341
    Nif = fftw_fft2((1.0 / sample) ** 2, My, Mx)              # :343
    MF = Mx * My
    k_inv = 1.0 / (k ** 2)                                     # :357
    ri, ci = conv_index(Mx, My)
    E = Nf[ri, ci]                                             # A[0]
    K = Nif[ri, ci]
    j = np.arange(MF)
    upj = lat.up[j % Mx].astype(np.complex128)
    wqj = lat.wq[j // Mx].astype(np.complex128)
    A1 = K * upj[None, :]
    A2 = K * wqj[None, :]
    up_r = upj                                                 # row r has pi = r % Mx
    wq_r = wqj
    P = np.zeros((4 * MF, 4 * MF), dtype=np.complex128)
    rr = np.arange(MF)
    P[0:MF, 2 * MF:3 * MF] = (up_r * k_inv)[:, None] * A2       # :378
    P[0:MF, 3 * MF:4 * MF] = (-up_r * k_inv)[:, None] * A1      # :379
    P[rr, 3 * MF + rr] += 1                                    # :380
    P[MF:2 * MF, 2 * MF:3 * MF] = (wq_r * k_inv)[:, None] * A2  # :382
    P[MF:2 * MF, 3 * MF:4 * MF] = (-wq_r * k_inv)[:, None] * A1  # :383
    P[MF + rr, 2 * MF + rr] += -1                              # :384
    P[2 * MF:3 * MF, MF:2 * MF] = -E                            # :386
    P[2 * MF + rr, rr] += -up_r * wq_r * k_inv                  # :387
    P[2 * MF + rr, MF + rr] += up_r * up_r * k_inv              # :388
    P[3 * MF:4 * MF, 0:MF] = E                                  # :390
    P[3 * MF + rr, rr] += -wq_r * wq_r * k_inv                  # :391
    P[3 * MF + rr, MF + rr] += up_r * wq_r * k_inv              # :392
    return P, Nf, Nif


# --------------------------------------------------------------------------
# a7/a8: eigensolve + sort/pair (third_Lapack.h:37-44, ScatterVolume.cpp:177-230)
# --------------------------------------------------------------------------
def mkl_eigensolve(A: np.ndarray):
    """third_Lapack.h:37-44: zgeev('N','V') -> eigenvalues, right eigenvectors."""
    w, v = sla.eig(A, left=False, right=True, check_finite=False)
    return w.astype(np.complex128), v.astype(np.complex128)


def _sorter_cmp(a, b):
    """ScatterVolume.cpp:177-184 as a three-way comparison."""
    va, vb = a[1], b[1]
    if abs(va.imag - vb.imag) > DBL_EPS:
        less = va.imag < vb.imag
    elif abs(va.real - vb.real) > DBL_EPS:
        less = va.real < vb.real
    else:
        less = va.imag < vb.imag
    if less:
        return -1
    # std::sort only needs `less`; emulate strict weak ordering
    if abs(va.imag - vb.imag) > DBL_EPS:
        more = vb.imag < va.imag
    elif abs(va.real - vb.real) > DBL_EPS:
        more = vb.real < va.real
    else:
        more = vb.imag < va.imag
    return 1 if more else 0


def eigen_sort(evl: np.ndarray, evt: np.ndarray):
    """ScatterVolume.cpp:190-230: sort by Im, then interleave largest-Im (even) / smallest-Im (odd)."""
    n = evl.size
    order = sorted(enumerate(evl), key=functools.cmp_to_key(_sorter_cmp))
    idx = [i for i, _ in order]
    out_l = np.empty(n, dtype=np.complex128)
    out_v = np.empty((n, n), dtype=np.complex128)
    for i in range(n // 2):
        out_l[2 * i] = evl[idx[n - 1 - i]]
        out_v[:, 2 * i] = evt[:, idx[n - 1 - i]]
        out_l[2 * i + 1] = evl[idx[i]]
        out_v[:, 2 * i + 1] = evt[:, idx[i]]
    return out_l, out_v


def mkl_inverse(A):
    """third_Lapack.h:56-63: zgesv against the identity."""
    return sla.solve(A, np.eye(A.shape[0], dtype=np.complex128), check_finite=False)


# --------------------------------------------------------------------------
# CLI parameters (ScatterVolume.cpp:511-529) and the solve driver
# --------------------------------------------------------------------------
@dataclass
class Params:
    """scattervolume options, same names and defaults (ScatterVolume.cpp:511-529)."""
    lambda_: float = 1.0
    direction: tuple = (0.0, 0.0, 1.0)
    ex: tuple = (0.0, 0.0)
    ey: tuple = (1.0, 0.0)
    ez: tuple = (0.0, 0.0)
    n: tuple = (1.0, 1.0)
    kappa: tuple = (0.0,)
    size: tuple = (10.0, 10.0, 2.0)
    z: float = 0.0
    coef: tuple = ()
    psf: bool = False
    external: bool = False
    npz: bool = False


def clamp_orders(M, num_pixels, p: Params, dirv):
    """ScatterVolume.cpp:599-651: order choice + evanescent clamp + pixel clamp.

    Returns (M, messages) where messages are the stdout warnings printed.
    """
    msgs = []
    in_coeff = list(p.coef)
    M = [0, 0]
    if len(in_coeff) == 0:
        M[0], M[1] = num_pixels[2], num_pixels[1]
    elif len(in_coeff) == 1:
        M[0] = M[1] = int(math.sqrt(in_coeff[0]))
    elif len(in_coeff) == 2:
        M[0], M[1] = int(in_coeff[0]), int(in_coeff[1])
    lam, size, n = p.lambda_, p.size, p.n
    if ((M[0] // 2) / size[0] * lam + dirv[0]) ** 2 + ((M[1] // 2) / size[1] * lam + dirv[1]) ** 2 >= n[0] ** 2:
        msgs.append("Cutting off invalid waves with imagnery sz...")
        if M[0] != 1 and M[1] != 1:
            if (M[0] // 2) / size[0] * lam + dirv[0] > 0.71 * n[0]:
                M[0] = int(0.707 * n[0] * 2 * size[0] / lam) - 1
                msgs.append(f"M[0] is corrected as {M[0]}")
            if (M[1] // 2) / size[1] * lam + dirv[1] > 0.71 * n[0]:
                M[1] = int(0.707 * n[1] * 2 * size[1] / lam) - 1
                msgs.append(f"M[1] is corrected as {M[1]}")
        if M[0] == 1:
            if (M[1] // 2) / size[1] * lam + abs(dirv[1]) >= n[0]:
                M[1] = int(n[1] * 2 * size[1] / lam - 1e-10)
                if M[1] % 2 == 0:
                    M[1] -= 1
        if M[1] == 1:
            if (M[0] // 2) / size[1] * lam + abs(dirv[0]) >= n[0]:
                M[0] = int(n[0] * 2 * size[0] / lam - 1e-10)
                if M[0] % 2 == 0:
                    M[0] -= 1
    if M[0] > num_pixels[2]:
        M[0] = num_pixels[2]
    if M[1] > num_pixels[1]:
        M[1] = num_pixels[1]
    return M, msgs


@dataclass
class Solution:
    """Everything the reference computes for one scattervolume run."""
    M: tuple
    k: float
    dirv: np.ndarray
    E0: np.ndarray
    z: np.ndarray
    Sx: np.ndarray
    Sy: np.ndarray
    Sz0: np.ndarray
    Sz1: np.ndarray
    EF: np.ndarray
    x: np.ndarray                      # [R_x R_y R_z T_x T_y T_z] (6 MF)
    Nf: list = field(default_factory=list)
    Nif: list = field(default_factory=list)
    eigenvalues: list = field(default_factory=list)
    eigenvectors: list = field(default_factory=list)
    Beta: list = field(default_factory=list)
    Q_check: list = field(default_factory=list)
    Q_hat: list = field(default_factory=list)
    msgs: list = field(default_factory=list)


def setup(sample: np.ndarray, p: Params):
    """ScatterVolume.cpp:573-651: direction, polarisation, k, layers, z planes, orders."""
    d = np.array(p.direction, dtype=np.float64)
    d = d / np.linalg.norm(d)                                           # :576
    e = np.array([complex(*p.ex), complex(*p.ey), complex(*p.ez)])
    e = orthogonalize(e, d)                                             # :582
    dirv = d * p.n[0]                                                   # :583
    k = 2 * PI / p.lambda_                                              # :586
    ni = [complex(p.n[0], 0.0), complex(p.n[1], p.kappa[0])]            # :154-159
    slices, num_pixels = reformat(sample)                               # :592
    Z = num_pixels[0]
    zz = np.empty(Z + 1)
    zz[0] = p.z - p.size[2] / 2.0                                       # :164
    for i in range(1, Z + 1):
        zz[i] = zz[i - 1] + p.size[2] / num_pixels[0]                   # :166
    M, msgs = clamp_orders(None, num_pixels, p, dirv)
    return d, e, dirv, k, ni, slices, num_pixels, zz, M, msgs


def solve(sample: np.ndarray, p: Params, keep=True) -> Solution:
    """ScatterVolume.cpp:506-987 (everything up to the .cw save)."""
    d, e, dirv, k, ni, slices, num_pixels, z, M, msgs = setup(sample, p)
    Mx, My = M
    MF = Mx * My
    Z = num_pixels[0]
    ZL = Z + 1
    kc = complex(k, 0.0)
    lat = upwq_cal(M, p.size, dirv, k, ni)
    # CalculateD (FourierWave.h:303-315)
    Phis, Nfs, Nifs = [], [], []
    for s in slices:
        P, Nf, Nif = phi(s, M, lat, k)
        Phis.append(P)
        Nfs.append(Nf)
        Nifs.append(Nif)
    # incident spectrum (:661-679)
    E0 = e
    Ef = []
    for c in range(3):
        if p.psf:
            Ef.append(E0[c] * np.ones((Mx, My), dtype=np.complex128))
        else:
            Ef.append(fftw_fft2(E0[c] * np.ones((num_pixels[1], num_pixels[2]), dtype=np.complex128), My, Mx))
    EF = np.concatenate([f.ravel(order="F") for f in Ef])
    Sx = lat.meshS0.ravel(order="F")                                    # :682-685
    Sy = lat.meshS1.ravel(order="F")
    Sz0 = lat.Sz[0].ravel(order="F")
    Sz1 = lat.Sz[1].ravel(order="F")
    # InitMatrices + SetGaussianConstraints (:148-151, 398-414)
    A = np.zeros((6 * MF, 6 * MF), dtype=np.complex128)
    b = np.zeros(6 * MF, dtype=np.complex128)
    m = np.arange(MF)
    A[m, m] = Sx
    A[m, MF + m] = Sy
    A[m, 2 * MF + m] = -Sz0
    A[MF + m, 3 * MF + m] = Sx
    A[MF + m, 4 * MF + m] = Sy
    A[MF + m, 5 * MF + m] = Sz1
    # EigenDecompositionD (:235-337)
    eigenvalues, eigenvectors, GD, GC = [], [], [], []
    for i in range(Z):
        evl, evt = mkl_eigensolve(Phis[i])
        sl, sv = eigen_sort(evl, evt)
        eigenvalues.append(sl)
        eigenvectors.append(sv)
        Phis[i] = None
    Gd_static = Gc_static = None
    for i in range(Z):
        lam = eigenvalues[i]
        if Z == 1:                                                      # :298-301
            dz_c, dz_d = z[ZL - 1] - z[0], z[0] - z[ZL - 1]
        else:                                                           # :303-306
            dz_c, dz_d = z[i + 1] - z[i], z[i] - z[i + 1]
        Ci = np.exp(1j * kc * lam * dz_c)
        Di = np.exp(1j * kc * lam * dz_d)
        V = eigenvectors[i]
        odd = (np.arange(4 * MF) % 2) != 0
        dG = np.where(odd, Di, 1.0)
        cG = np.where(odd, 1.0, Ci)
        Gd = V * dG[None, :]
        Gc = V * cG[None, :]
        if not p.external:
            GD.append(Gd)
            GC.append(Gc)
        if i == 0:
            Gd_static, Gc_static = Gd, Gc
        else:
            tmp = mkl_inverse(Gd)
            tmp2 = Gc @ tmp
            Gc_static = tmp2 @ Gc_static
    # MatTransfer (:339-395)
    phase = np.exp(1j * kc * z[0] * Sz0)
    I = np.eye(MF, dtype=np.complex128)
    dg = np.diag
    f1 = np.zeros((4 * MF, 3 * MF), dtype=np.complex128)
    f2 = np.zeros_like(f1)
    f3 = np.zeros_like(f1)
    f1[0:MF, 0:MF] = dg(phase)
    f1[MF:2 * MF, MF:2 * MF] = dg(phase)
    f1[2 * MF:3 * MF, MF:2 * MF] = -dg(phase * Sz0)
    f1[2 * MF:3 * MF, 2 * MF:3 * MF] = dg(phase * Sy)
    f1[3 * MF:4 * MF, 0:MF] = dg(phase * Sz0)
    f1[3 * MF:4 * MF, 2 * MF:3 * MF] = -dg(phase * Sx)
    f2[0:MF, 0:MF] = I
    f2[MF:2 * MF, MF:2 * MF] = I
    f2[2 * MF:3 * MF, MF:2 * MF] = dg(Sz0)
    f2[2 * MF:3 * MF, 2 * MF:3 * MF] = dg(Sy)
    f2[3 * MF:4 * MF, 0:MF] = -dg(Sz0)
    f2[3 * MF:4 * MF, 2 * MF:3 * MF] = -dg(Sx)
    f3[0:MF, 0:MF] = -I
    f3[MF:2 * MF, MF:2 * MF] = -I
    f3[2 * MF:3 * MF, MF:2 * MF] = dg(Sz1)
    f3[2 * MF:3 * MF, 2 * MF:3 * MF] = -dg(Sy)
    f3[3 * MF:4 * MF, 0:MF] = -dg(Sz1)
    f3[3 * MF:4 * MF, 2 * MF:3 * MF] = dg(Sx)
    # SetBoundaryConditions (:417-466)
    Gc_inv = mkl_inverse(Gc_static)
    A[2 * MF:6 * MF, 0:3 * MF] = f2
    tmp = Gd_static @ Gc_inv
    A[2 * MF:6 * MF, 3 * MF:6 * MF] = tmp @ f3
    b[2 * MF:6 * MF] = -(f1 @ EF)
    # MKL_linearsolve (:739)
    x = sla.solve(A, b, check_finite=False)
    sol = Solution(M=(Mx, My), k=k, dirv=dirv, E0=E0, z=z, Sx=Sx, Sy=Sy, Sz0=Sz0, Sz1=Sz1,
                   EF=EF, x=x, msgs=msgs)
    if keep:
        sol.Nf, sol.Nif = Nfs, Nifs
    sol.eigenvalues = eigenvalues
    sol.eigenvectors = eigenvectors
    if p.external:
        return sol
    # Beta chain (:753-797)
    Beta = []
    beta = None
    for i in range(Z):
        if i == 0:
            tmp = mkl_inverse(GD[0])
            beta = (tmp @ f1) @ EF
            beta = beta + (tmp @ f2) @ x[0:3 * MF]
        else:
            tmp = mkl_inverse(GD[i])
            beta = (tmp @ GC[i - 1]) @ beta
        Beta.append(beta)
    sol.Beta = Beta
    # Q_check / Q_hat + Pz (:802-889)
    q_series = lin_spaced(My, -float(My // 2), float((My - 1) // 2))
    p_series = lin_spaced(Mx, -float(Mx // 2), float((Mx - 1) // 2))
    WQ = 2.0 * q_series * M_PI / p.size[1]
    UP = 2.0 * p_series * M_PI / p.size[0]
    j = np.arange(MF)
    up_j = UP[j % Mx] + dirv[0] * kc
    wq_j = WQ[j // Mx] + dirv[1] * kc
    # Pz lookup: linear index ((indR+My/2)%My)*Mx + (indC+Mx/2)%Mx into the
    # column-major (My x Mx) storage of NIf (ScatterVolume.cpp:872)
    ri, ci = conv_index(Mx, My)
    lin = ri * Mx + ci
    Q_check, Q_hat = [], []
    for i in range(Z):
        V = eigenvectors[i]
        Vev, Vod = V[:, 0::2], V[:, 1::2]
        Q1 = Vev * Beta[i][0::2][None, :]
        Q2 = Vod * Beta[i][1::2][None, :]
        Qc = np.zeros((3 * MF, 2 * MF), dtype=np.complex128)
        Qh = np.zeros((3 * MF, 2 * MF), dtype=np.complex128)
        Qc[0:2 * MF] = Q1[0:2 * MF]
        Qh[0:2 * MF] = Q2[0:2 * MF]
        if not p.npz:
            KP = Nifs[i].ravel(order="F")[lin]
            I1, J1 = Q1[2 * MF:3 * MF], Q1[3 * MF:4 * MF]
            I2, J2 = Q2[2 * MF:3 * MF], Q2[3 * MF:4 * MF]
            Qc[2 * MF:3 * MF] += (-1.0 / kc) * (KP @ (up_j[:, None] * J1 - wq_j[:, None] * I1))
            Qh[2 * MF:3 * MF] += (-1.0 / kc) * (KP @ (up_j[:, None] * J2 - wq_j[:, None] * I2))
        Q_check.append(Qc)
        Q_hat.append(Qh)
    sol.Q_check, sol.Q_hat = Q_check, Q_hat
    return sol


# --------------------------------------------------------------------------
# the chain split by layer blocks (ScatterVolume.cpp:282-336 over a layer
# range) and the boundary step from a given chain (:339-466, 739)
# --------------------------------------------------------------------------
def chain_block(sample: np.ndarray, p: Params, lb: int, le: int):
    """Ordered product of the transfer matrices of layers [lb, le) and, for lb == 0, GD_0.

    Gc_static <- Gc_i inv(Gd_i) Gc_static (:326-335) restricted to the block:
    P = T_{le-1} ... T_{lb} with T_i = Gc_i inv(Gd_i), and Gc_0 in place of T_0
    when the block starts at layer 0 (Gc_static starts as Gc_0, :321-324).
    """
    d, e, dirv, k, ni, slices, num_pixels, z, M, msgs = setup(sample, p)
    Mx, My = M
    MF = Mx * My
    Z = num_pixels[0]
    ZL = Z + 1
    kc = complex(k, 0.0)
    lat = upwq_cal(M, p.size, dirv, k, ni)
    P = None
    Gd0 = None
    for i in range(lb, le):
        Phi, _, _ = phi(slices[i], M, lat, k)
        lam, V = eigen_sort(*mkl_eigensolve(Phi))
        if Z == 1:                                                      # :298-301
            dz_c, dz_d = z[ZL - 1] - z[0], z[0] - z[ZL - 1]
        else:                                                           # :303-306
            dz_c, dz_d = z[i + 1] - z[i], z[i] - z[i + 1]
        odd = (np.arange(4 * MF) % 2) != 0
        Gd = V * np.where(odd, np.exp(1j * kc * lam * dz_d), 1.0)[None, :]
        Gc = V * np.where(odd, 1.0, np.exp(1j * kc * lam * dz_c))[None, :]
        if i == 0:
            Gd0 = Gd
            T = Gc
        else:
            T = Gc @ mkl_inverse(Gd)
        P = T if P is None else T @ P
    return P, Gd0


def boundary_from_chain(sample: np.ndarray, p: Params, Gc_static, Gd_static):
    """x = [R; T] from the whole chain: MatTransfer, SetBoundaryConditions and zgesv (:339-466, 739)."""
    d, e, dirv, k, ni, slices, num_pixels, z, M, msgs = setup(sample, p)
    Mx, My = M
    MF = Mx * My
    kc = complex(k, 0.0)
    lat = upwq_cal(M, p.size, dirv, k, ni)
    E0 = e
    Ef = []
    for c in range(3):
        if p.psf:
            Ef.append(E0[c] * np.ones((Mx, My), dtype=np.complex128))
        else:
            Ef.append(fftw_fft2(E0[c] * np.ones((num_pixels[1], num_pixels[2]), dtype=np.complex128), My, Mx))
    EF = np.concatenate([f.ravel(order="F") for f in Ef])
    Sx = lat.meshS0.ravel(order="F")
    Sy = lat.meshS1.ravel(order="F")
    Sz0 = lat.Sz[0].ravel(order="F")
    Sz1 = lat.Sz[1].ravel(order="F")
    A = np.zeros((6 * MF, 6 * MF), dtype=np.complex128)
    b = np.zeros(6 * MF, dtype=np.complex128)
    m = np.arange(MF)
    A[m, m] = Sx
    A[m, MF + m] = Sy
    A[m, 2 * MF + m] = -Sz0
    A[MF + m, 3 * MF + m] = Sx
    A[MF + m, 4 * MF + m] = Sy
    A[MF + m, 5 * MF + m] = Sz1
    phase = np.exp(1j * kc * z[0] * Sz0)
    I = np.eye(MF, dtype=np.complex128)
    dg = np.diag
    f1 = np.zeros((4 * MF, 3 * MF), dtype=np.complex128)
    f2 = np.zeros_like(f1)
    f3 = np.zeros_like(f1)
    f1[0:MF, 0:MF] = dg(phase)
    f1[MF:2 * MF, MF:2 * MF] = dg(phase)
    f1[2 * MF:3 * MF, MF:2 * MF] = -dg(phase * Sz0)
    f1[2 * MF:3 * MF, 2 * MF:3 * MF] = dg(phase * Sy)
    f1[3 * MF:4 * MF, 0:MF] = dg(phase * Sz0)
    f1[3 * MF:4 * MF, 2 * MF:3 * MF] = -dg(phase * Sx)
    f2[0:MF, 0:MF] = I
    f2[MF:2 * MF, MF:2 * MF] = I
    f2[2 * MF:3 * MF, MF:2 * MF] = dg(Sz0)
    f2[2 * MF:3 * MF, 2 * MF:3 * MF] = dg(Sy)
    f2[3 * MF:4 * MF, 0:MF] = -dg(Sz0)
    f2[3 * MF:4 * MF, 2 * MF:3 * MF] = -dg(Sx)
    f3[0:MF, 0:MF] = -I
    f3[MF:2 * MF, MF:2 * MF] = -I
    f3[2 * MF:3 * MF, MF:2 * MF] = dg(Sz1)
    f3[2 * MF:3 * MF, 2 * MF:3 * MF] = -dg(Sy)
    f3[3 * MF:4 * MF, 0:MF] = -dg(Sz1)
    f3[3 * MF:4 * MF, 2 * MF:3 * MF] = dg(Sx)
    A[2 * MF:6 * MF, 0:3 * MF] = f2
    A[2 * MF:6 * MF, 3 * MF:6 * MF] = (Gd_static @ mkl_inverse(Gc_static)) @ f3
    b[2 * MF:6 * MF] = -(f1 @ EF)
    return sla.solve(A, b, check_finite=False)


# --------------------------------------------------------------------------
# a16/a17: wave lists of the coupled-wave structure (ScatterVolume.cpp:469-493, 907-987)
# --------------------------------------------------------------------------
def wind(E, kvec, dz):
    """tira::planewave::wind(0, 0, dz): E0 <- E0 exp(i kz dz) (E = E0 e^{i k.r} convention)."""
    return E * np.exp(1j * kvec[..., 2] * dz)[..., None]


@dataclass
class WaveSet:
    """Plane waves grouped like CoupledWaveStructure (E has 3 components, k has 3)."""
    Pi_E: np.ndarray
    Pi_k: np.ndarray
    z: np.ndarray                  # boundary z (ZL,)
    Pr_E: list
    Pr_k: list
    Pt_E: list
    Pt_k: list


def build_waves(sol: Solution, p: Params) -> WaveSet:
    """ScatterVolume.cpp:907-987 vectorised.  Keeps the solver's Ez (Pz)."""
    Mx, My = sol.M
    MF = Mx * My
    k = complex(sol.k, 0.0)
    Z = len(sol.eigenvalues)
    ZL = Z + 1
    pidx = np.arange(MF)          # p = kk*Mx + j over the loops kk, j
    Sx, Sy, Sz0, Sz1, EF, x = sol.Sx, sol.Sy, sol.Sz0, sol.Sz1, sol.EF, sol.x
    kx = Sx[pidx] * k
    ky = Sy[pidx] * k
    Pi_k = np.stack([kx, ky, Sz0[pidx] * k], axis=-1)
    Pi_E = np.stack([EF[pidx], EF[MF + pidx], EF[2 * MF + pidx]], axis=-1)
    r_k = np.stack([kx, ky, -Sz0[pidx] * k * p.n[0]], axis=-1)           # :474-480
    r_E = np.stack([x[pidx], x[MF + pidx], x[2 * MF + pidx]], axis=-1)
    t_k = np.stack([kx, ky, Sz1[pidx] * k * p.n[1]], axis=-1)            # :481-487
    t_E = np.stack([x[3 * MF + pidx], x[4 * MF + pidx], x[5 * MF + pidx]], axis=-1)
    zs = np.zeros(ZL)
    Pr_E, Pr_k, Pt_E, Pt_k = [], [], [], []

    def internal(l_eig, Q, parity, zl):
        lam = sol.eigenvalues[l_eig][parity::2]            # (2MF,)
        kk = np.empty((MF, 2 * MF, 3), dtype=np.complex128)
        kk[..., 0] = kx[:, None]
        kk[..., 1] = ky[:, None]
        kk[..., 2] = (lam * k)[None, :]
        EE = np.stack([Q[pidx, :], Q[MF + pidx, :], Q[2 * MF + pidx, :]], axis=-1)
        EE = wind(EE, kk, -zl)
        return EE.reshape(-1, 3), kk.reshape(-1, 3)

    for l in range(ZL):
        empty = (np.zeros((0, 3), np.complex128), np.zeros((0, 3), np.complex128))
        if l == 0:
            zs[l] = sol.z[l]
            pr = (wind(r_E, r_k, -sol.z[l]), r_k)
            pt = internal(0, sol.Q_check[0], 0, sol.z[l]) if not p.external else empty
        elif l == ZL - 1:
            zs[l] = sol.z[l]
            pt = (wind(t_E, t_k, -sol.z[l]), t_k)
            pr = internal(l - 1, sol.Q_hat[l - 1], 1, sol.z[l]) if not p.external else empty
        else:
            if not p.external:
                pr = internal(l - 1, sol.Q_hat[l - 1], 1, sol.z[l])
                pt = internal(l, sol.Q_check[l], 0, sol.z[l])
                zs[l] = sol.z[l]
            else:
                pr = pt = empty
        Pr_E.append(pr[0])
        Pr_k.append(pr[1])
        Pt_E.append(pt[0])
        Pt_k.append(pt[1])
    return WaveSet(Pi_E, Pi_k, zs, Pr_E, Pr_k, Pt_E, Pt_k)


def transverse_ez(E, kv):
    """E_z rebuilt from (Ex, Ey, k) by transversality, the assumed tira::planewave::getE0()."""
    E = E.copy()
    E[:, 2] = -(kv[:, 0] * E[:, 0] + kv[:, 1] * E[:, 1]) / kv[:, 2]
    return E
