"""Coupled-wave (.cw) files in the reference's byte layout and record frame.

Layout (CoupledWaveStructure.h:63-125): u64 sizeof(double) = 8; u64 #Pi, the
incident records; u64 #layers; per layer: f64 z, u64 #Pr, records, u64 #Pt,
records.  One record = sizeof(tira::planewave<double>) = 80 bytes =
{E0x, E0y, kx, ky, kz} complex128.

Record frame: tira's planewave keeps E0 in a frame whose z axis is the real
propagation direction Re(k)/|Re(k)| (the minimal rotation taking z-hat
there), and the file stores the first two components of E0 in that frame.
getE0() rebuilds the third from k . E = 0 in the same frame.  This reading
reproduces every record of the reference's shipped data/psf.cw and the
incident and transmitted records of x64/a.cw from their restated solves.

Downward waves made by tira::planewave's constructor from a Cartesian E0 (the
reflected waves of ScatterLayer.cpp:246-251) hold their pair in the frame of
the z-mirrored direction (Re kx, Re ky, -Re kz) instead: with mirror_down=True
every record of x64/a.cw, the reflected ones included, is reproduced, and its
field is continuous at every interface (read in the wave's own frame it jumps
by up to 15 %).  Waves made by tira's scatter() (ScatterPlane.cpp:175, 244)
keep their own frame (psf.cw's reflected records are 4 % off when mirrored).
"""
from __future__ import annotations

import struct

import numpy as np


def frames(k, mirror_down: bool = False):
    """(N, 3, 3) rotations whose third column is Re(k)/|Re(k)| (minimal rotation from z-hat); with mirror_down,
    a wave with Re kz < 0 takes the rotation of its z-mirrored direction."""
    kr = np.real(np.asarray(k, dtype=np.complex128)).reshape(-1, 3)
    if mirror_down:
        kr = kr.copy()
        kr[:, 2] = np.abs(kr[:, 2])
    kh = kr / np.linalg.norm(kr, axis=1, keepdims=True)
    ax0, ax1, c = -kh[:, 1], kh[:, 0], kh[:, 2]
    s2 = ax0 * ax0 + ax1 * ax1
    small = s2 < 1e-30
    f = np.where(small, 0.0, (1.0 - c) / np.where(small, 1.0, s2))
    R = np.zeros((len(kh), 3, 3))
    R[:, 0, 0] = 1.0 - f * ax1 * ax1
    R[:, 0, 1] = f * ax0 * ax1
    R[:, 0, 2] = ax1
    R[:, 1, 0] = f * ax0 * ax1
    R[:, 1, 1] = 1.0 - f * ax0 * ax0
    R[:, 1, 2] = -ax0
    R[:, 2, 0] = -ax1
    R[:, 2, 1] = ax0
    R[:, 2, 2] = c
    down = small & (c < 0)                       # straight down: half turn about x
    R[small] = np.eye(3)
    R[down] = np.diag([1.0, -1.0, -1.0])
    return R


def to_record(E, k, mirror_down: bool = False):
    """Cartesian E0 (N, 3) -> the stored pair (N, 2)."""
    R = frames(k, mirror_down)
    return np.einsum("nij,ni->nj", R, np.asarray(E, dtype=np.complex128).reshape(-1, 3))[:, :2]


def from_record(E2, k, mirror_down: bool = False):
    """Stored pair (N, 2) -> Cartesian E0 (N, 3), the third local component from k . E = 0."""
    k = np.asarray(k, dtype=np.complex128).reshape(-1, 3)
    E2 = np.asarray(E2, dtype=np.complex128).reshape(-1, 2)
    R = frames(k, mirror_down)
    kp = np.einsum("nij,ni->nj", R, k)
    ez = np.where(kp[:, 2] != 0, -(kp[:, 0] * E2[:, 0] + kp[:, 1] * E2[:, 1]) / np.where(kp[:, 2] != 0, kp[:, 2], 1),
                  0)
    loc = np.stack([E2[:, 0], E2[:, 1], ez], 1)
    return np.einsum("nij,nj->ni", R, loc)


def _records(E, k, mirror_down=False):
    E = np.asarray(E, dtype=np.complex128).reshape(-1, 3)
    rec = np.empty((len(E), 5), dtype=np.complex128)
    if len(E):
        rec[:, 0:2] = to_record(E, k, mirror_down)
        rec[:, 2:5] = np.asarray(k, dtype=np.complex128).reshape(-1, 3)
    return rec.tobytes()


def save(path, Pi_E, Pi_k, layers, mirror_down: bool = False):
    """Write a .cw file.  E arguments are Cartesian E0 (N, 3); layers = [(z, Pr_E, Pr_k, Pt_E, Pt_k)];
    mirror_down: downward waves' pairs in the mirrored frame, as the reference's scatterlayer writes them."""
    with open(path, "wb") as f:
        f.write(struct.pack("<QQ", 8, len(Pi_E)))
        f.write(_records(Pi_E, Pi_k, mirror_down))
        f.write(struct.pack("<Q", len(layers)))
        for z, PrE, Prk, PtE, Ptk in layers:
            f.write(struct.pack("<dQ", float(z), len(PrE)))
            f.write(_records(PrE, Prk, mirror_down))
            f.write(struct.pack("<Q", len(PtE)))
            f.write(_records(PtE, Ptk, mirror_down))


def _read_raw(path):
    """(Pi pairs, Pi k, [(z, Pr pairs, Pr k, Pt pairs, Pt k)]) as stored."""
    b = open(path, "rb").read()
    sz, npi = struct.unpack_from("<QQ", b, 0)
    if sz != 8:
        raise ValueError("only double-precision .cw files are supported")
    o = 16

    def recs(count):
        nonlocal o
        r = np.frombuffer(b, dtype=np.complex128, count=5 * count, offset=o).reshape(count, 5)
        o += 80 * count
        return r[:, 0:2].copy(), r[:, 2:5].copy()

    Pi = recs(npi)
    (nl,) = struct.unpack_from("<Q", b, o)
    o += 8
    layers = []
    for _ in range(nl):
        z, npr = struct.unpack_from("<dQ", b, o)
        o += 16
        Pr = recs(npr)
        (npt,) = struct.unpack_from("<Q", b, o)
        o += 8
        Pt = recs(npt)
        layers.append((z,) + Pr + Pt)
    return Pi, layers


def interface_jump(Pi, layers, mirror_down: bool, points: int = 8) -> float:
    """Largest jump of the tangential (x, y) field across the first interface, relative to the field there, with
    the stored pairs read in the given frame: the plane-wave sum of region 0 (incident + reflected at z_0)
    against that of region 1 (transmitted at z_0 + reflected at z_1), both on the plane z = z_0 (the regions of
    cpuEvaluator.cpp:34-102).  The reading the file was written in gives a continuous field."""
    if not layers:
        return 0.0

    def waves(pk):
        E2, k = pk
        return (from_record(E2, k, mirror_down), k) if len(E2) else (np.zeros((0, 3), complex), k)
    z0 = layers[0][0]
    above = [waves(Pi), waves(layers[0][1:3])]
    below = [waves(layers[0][3:5])] + ([waves(layers[1][1:3])] if len(layers) > 1 else [])
    kmax = max([np.abs(k).max() for _, k in above + below if len(k)] + [1.0])
    rng = np.random.default_rng(0)
    xy = rng.uniform(-1.0, 1.0, (points, 2)) * (2 * np.pi / kmax)
    r = np.c_[xy, np.full(points, z0)]

    def field(parts):
        out = np.zeros((points, 3), complex)
        for E, k in parts:
            if len(E):
                out += np.exp(1j * (r @ k.T)) @ E
        return out
    a, b = field(above)[:, :2], field(below)[:, :2]
    scale = max(np.abs(a).max(), np.abs(b).max())
    return float(np.abs(a - b).max() / scale) if scale > 0 else 0.0


def detect_mirror_down(path) -> bool:
    """Which record frame a file's downward waves were written in, from the physics: True when reading them in
    the z-mirrored direction's frame makes the field continuous across the first interface and the own frame
    does not (the reference's scatterlayer files), False otherwise (its scatterplane files, this package's)."""
    Pi, layers = _read_raw(path)
    return interface_jump(Pi, layers, True) < interface_jump(Pi, layers, False)


def load(path, mirror_down=False):
    """Read a .cw file: (Pi_E, Pi_k, layers) with Cartesian E0 (N, 3) as getE0() rebuilds it.  mirror_down: True
    for files whose downward waves hold mirrored-frame pairs (the reference's scatterlayer output), "auto" to
    decide from the field's continuity at the first interface (detect_mirror_down)."""
    Pi, raw = _read_raw(path)
    if mirror_down == "auto":
        mirror_down = interface_jump(Pi, raw, True) < interface_jump(Pi, raw, False)

    def conv(E2, k):
        return from_record(E2, k, bool(mirror_down)) if len(E2) else np.zeros((0, 3), np.complex128)
    layers = [(z, conv(a, ak), ak, conv(c, ck), ck) for z, a, ak, c, ck in raw]
    return conv(*Pi), Pi[1], layers
