"""Oracle: .cw file format, wave unpacking and the field evaluator (test infrastructure only).

* ``save``/``load`` restate ``CoupledWaveStructure<T>::save/load``
  (CoupledWaveStructure.h:63-125) with the record size pinned by the two
  files the reference ships (``data/psf.cw``, ``x64/a.cw``): one record is
  ``sizeof(tira::planewave<double>)`` = 80 bytes = {E0x, E0y, kx, ky, kz}
  complex128.  E0z is not stored.
* ``get_e0_tira``/``put_e0_tira``: the storage frame of a record's E pair
  (tira's planewave keeps E in a frame rotated to the real k direction),
  pinned by reproducing both shipped files from their incident waves.
* ``unpack`` restates ``cw_allocate``/``cw_unpack`` (cpuEvaluator.cpp:34-102):
  region 0 = Pi + Pr_0, region l = Pt_{l-1} + Pr_l, last = Pt_last.
* ``evaluate`` restates the GPU ``evaluate`` device function
  (gpuEvaluator.cu:28-68) -- layer lookup ``z >= z_l - 0.001`` then the plane
  wave sum -- in float64 (the reference sums in float32; the float32 form is
  ``evaluate_f32``).
"""
from __future__ import annotations

import struct

import numpy as np

REC = 80  # bytes per plane-wave record


def save(path, Pi_E, Pi_k, layers):
    """CoupledWaveStructure.h:63-92.  layers = [(z, Pr_E, Pr_k, Pt_E, Pt_k)]."""
    with open(path, "wb") as f:
        f.write(struct.pack("<Q", 8))
        f.write(struct.pack("<Q", len(Pi_E)))
        f.write(_records(Pi_E, Pi_k))
        f.write(struct.pack("<Q", len(layers)))
        for z, PrE, Prk, PtE, Ptk in layers:
            f.write(struct.pack("<d", z))
            f.write(struct.pack("<Q", len(PrE)))
            f.write(_records(PrE, Prk))
            f.write(struct.pack("<Q", len(PtE)))
            f.write(_records(PtE, Ptk))


def _records(E, k):
    E = np.asarray(E, dtype=np.complex128)
    E = E.reshape(len(E), -1) if len(E) else np.zeros((0, 3), np.complex128)
    k = np.asarray(k, dtype=np.complex128).reshape(-1, 3)
    rec = np.empty((len(E), 5), dtype=np.complex128)
    if len(E):
        rec[:, 0:2] = E[:, 0:2]
        rec[:, 2:5] = k
    return rec.tobytes()


def load(path):
    """CoupledWaveStructure.h:94-125.  Returns (Pi_E2, Pi_k, layers) with E holding (Ex, Ey)."""
    b = open(path, "rb").read()
    o = 0
    sz, npi = struct.unpack_from("<QQ", b, o)
    o += 16
    if sz != 8:
        raise ValueError("only double-precision .cw files are supported")

    def recs(n):
        nonlocal o
        r = np.frombuffer(b, dtype=np.complex128, count=n * 5, offset=o).reshape(n, 5)
        o += n * REC
        return r[:, 0:2].copy(), r[:, 2:5].copy()

    PiE, Pik = recs(npi)
    (nl,) = struct.unpack_from("<Q", b, o)
    o += 8
    layers = []
    for _ in range(nl):
        (z,) = struct.unpack_from("<d", b, o)
        o += 8
        (npr,) = struct.unpack_from("<Q", b, o)
        o += 8
        PrE, Prk = recs(npr)
        (npt,) = struct.unpack_from("<Q", b, o)
        o += 8
        PtE, Ptk = recs(npt)
        layers.append((z, PrE, Prk, PtE, Ptk))
    if o != len(b):
        raise ValueError(f"trailing bytes in {path}: parsed {o} of {len(b)}")
    return PiE, Pik, layers


def get_e0(E2, k):
    """Assumed tira::planewave::getE0(): Ez = -(kx Ex + ky Ey) / kz (transversality)."""
    E = np.zeros((len(E2), 3), dtype=np.complex128)
    E[:, 0:2] = E2[:, 0:2]
    E[:, 2] = -(k[:, 0] * E2[:, 0] + k[:, 1] * E2[:, 1]) / k[:, 2]
    return E


def tira_frame(k, mirror_down=False):
    """Rotation R whose third column is the real propagation direction Re(k)/|Re(k)|.

    R is the minimal (Rodrigues) rotation taking z-hat to that direction: about
    the axis z-hat x k-hat by the angle between them.  Straight down (-z-hat)
    has no minimal rotation; a half turn about x is used there (no shipped
    record is exactly vertical downwards, so that case is unpinned).

    mirror_down: for a downward wave (Re k_z < 0) the frame of the z-mirrored
    direction (Re k_x, Re k_y, -Re k_z) instead -- the frame of the records
    that tira::planewave's constructor makes from a Cartesian E0 and a
    downward k (the reflected waves of ScatterLayer.cpp:246-251, and by the
    same constructor those of ScatterVolume.cpp:469-493, 907-987).  Records of
    waves made by tira's scatter() (ScatterPlane.cpp:175, 244) keep their own
    frame.  Pinned by the shipped files: x64/a.cw's reflected records are the
    restated scatterlayer solve in the mirrored frame (~1e-15; its field is then
    continuous at every interface, and jumps by up to 15 % in the own frame),
    data/psf.cw's reflected records the restated scatterplane solve in the own
    frame (~1e-15; 4 % median off in the mirrored one).
    """
    kr = np.real(np.asarray(k, dtype=np.complex128))
    if mirror_down and kr[2] < 0:
        kr = kr * np.array([1.0, 1.0, -1.0])
    kh = kr / np.linalg.norm(kr)
    ax = np.array([-kh[1], kh[0], 0.0])           # z-hat x k-hat
    s2 = ax @ ax
    if s2 < 1e-30:
        return np.eye(3) if kh[2] > 0 else np.diag([1.0, -1.0, -1.0])
    K = np.array([[0.0, -ax[2], ax[1]], [ax[2], 0.0, -ax[0]], [-ax[1], ax[0], 0.0]])
    return np.eye(3) + K + (1.0 - kh[2]) / s2 * (K @ K)


def get_e0_tira(E2, k, mirror_down=False):
    """A record's E0 as tira::planewave::getE0() rebuilds it (pinned by the shipped files).

    A record stores (E0x, E0y) = the first two components of R^T E in the
    frame of ``tira_frame(k, mirror_down)``; the third local component is
    rebuilt from k . E = 0 in that frame (k' = R^T k, complex for absorbing
    media).  Under this reading every wave of data/psf.cw (scatterplane, 4096
    incident, reflected and transmitted records; own frame) and every wave of
    x64/a.cw (scatterlayer, three boundaries; mirror_down for its reflected
    records) is reproduced to ~1e-15 by the layer solve of
    ScatterLayer.cpp:152-266 fed with the file's own incident waves.
    """
    E2 = np.asarray(E2, dtype=np.complex128).reshape(-1, 2)
    k = np.asarray(k, dtype=np.complex128).reshape(-1, 3)
    out = np.zeros((len(E2), 3), dtype=np.complex128)
    for i in range(len(E2)):
        R = tira_frame(k[i], mirror_down)
        kp = R.T @ k[i]
        ez = -(kp[0] * E2[i, 0] + kp[1] * E2[i, 1]) / kp[2] if kp[2] != 0 else 0.0
        out[i] = R @ np.array([E2[i, 0], E2[i, 1], ez])
    return out


def put_e0_tira(E, k, mirror_down=False):
    """The (E0x, E0y) pair a record stores for a Cartesian E0 (inverse of get_e0_tira)."""
    E = np.asarray(E, dtype=np.complex128).reshape(-1, 3)
    k = np.asarray(k, dtype=np.complex128).reshape(-1, 3)
    out = np.zeros((len(E), 2), dtype=np.complex128)
    for i in range(len(E)):
        out[i] = (tira_frame(k[i], mirror_down).T @ E[i])[:2]
    return out


def unpack(Pi_E, Pi_k, layers):
    """cpuEvaluator.cpp:34-102.  Returns (z_layers, begin, end, W_E, W_k) with 3-component E."""
    zl = np.array([L[0] for L in layers], dtype=np.float64)
    begin, end = [0], []
    total = len(Pi_E)
    E_parts = [Pi_E]
    k_parts = [Pi_k]
    for (z, PrE, Prk, PtE, Ptk) in layers:
        total += len(PrE)
        end.append(total)
        begin.append(total)
        total += len(PtE)
        E_parts += [PrE, PtE]
        k_parts += [Prk, Ptk]
    end.append(total)
    WE = np.concatenate([np.asarray(e, dtype=np.complex128).reshape(-1, 3) for e in E_parts]) if total else np.zeros((0, 3), np.complex128)
    Wk = np.concatenate([np.asarray(k, dtype=np.complex128).reshape(-1, 3) for k in k_parts]) if total else np.zeros((0, 3), np.complex128)
    return zl, np.array(begin), np.array(end), WE, Wk


def region_of(z, z_layers, eps=0.001):
    """gpuEvaluator.cu:31-37 (eps = 0.001) / cpuEvaluator.cpp:301-306 (eps = 0)."""
    l = np.zeros(np.shape(z), dtype=np.int64)
    for li, zl in enumerate(z_layers):
        l = np.where(z >= zl - eps, li + 1, l)
    return l


def evaluate(points, z_layers, begin, end, WE, Wk, eps=0.001):
    """gpuEvaluator.cu:28-68 in float64.  points: (P, 3) -> E (P, 3) complex128."""
    pts = np.asarray(points, dtype=np.float64)
    reg = region_of(pts[:, 2], z_layers, eps)
    out = np.zeros((len(pts), 3), dtype=np.complex128)
    for l in np.unique(reg):
        sel = np.nonzero(reg == l)[0]
        b, e = int(begin[l]), int(end[l])
        if e <= b:
            continue
        K = Wk[b:e]
        E = WE[b:e]
        for c0 in range(0, len(sel), 4096):
            s = sel[c0:c0 + 4096]
            ph = np.exp(1j * (pts[s] @ K.T))          # (P, W)
            out[s] = ph @ E
    return out


def evaluate_f32(points, z_layers, begin, end, WE, Wk, eps=0.001):
    """gpuEvaluator.cu:28-68 with the reference's float32 arithmetic (complex64 terms)."""
    pts = np.asarray(points, dtype=np.float32)
    reg = region_of(pts[:, 2].astype(np.float64), z_layers.astype(np.float32).astype(np.float64), eps)
    out = np.zeros((len(pts), 3), dtype=np.complex64)
    K = Wk.astype(np.complex64)
    E = WE.astype(np.complex64)
    for l in np.unique(reg):
        sel = np.nonzero(reg == l)[0]
        b, e = int(begin[l]), int(end[l])
        if e <= b:
            continue
        for c0 in range(0, len(sel), 4096):
            s = sel[c0:c0 + 4096]
            kr = pts[s] @ K[b:e].T
            out[s] = np.exp(1j * kr).astype(np.complex64) @ E[b:e]
    return out


def slice_points(axis, center, extent, N, plane):
    """Grid of scatterview --nogui (ScatterView.cpp:354-370, 713-724).

    axis 1 -> x-z slice at y = plane, rows = z, cols = x (gpuEvaluator.cu:91-109).
    axis 2 -> x-y slice at z = plane; axis 0 -> y-z slice at x = plane.
    Returns (N*N, 3) points in the row-major order of the saved (N, N, 3) array.
    """
    d = extent / (N - 1)
    x0 = center[0] - extent / 2
    y0 = center[1] - extent / 2
    z0 = center[2] - extent / 2
    i = np.arange(N)
    if axis == 1:
        zz, xx = np.meshgrid(z0 + d * i, x0 + d * i, indexing="ij")
        return np.stack([xx.ravel(), np.full(N * N, plane), zz.ravel()], -1)
    if axis == 2:
        yy, xx = np.meshgrid(y0 + d * i, x0 + d * i, indexing="ij")
        return np.stack([xx.ravel(), yy.ravel(), np.full(N * N, plane)], -1)
    zz, yy = np.meshgrid(z0 + d * i, y0 + d * i, indexing="ij")
    return np.stack([np.full(N * N, plane), yy.ravel(), zz.ravel()], -1)
