"""Seeded synthetic samples with the shapes of the benchmark workloads.

The reference's sample scripts (data/*.py, cylindermaker.py) write complex128
refractive-index arrays, shape (Z, Y, X) or (Y, X); these generators produce
the same kind of array from ``numpy.random.default_rng(seed)``:

* ``triangle_map``   -- 64x64 map over a 10x10 um period, one random triangle
  of n = 1.4 in n = 1.0 (the thin-volume workload, M = 11x11).
* ``sphere_volume``  -- 128x128x32 voxels over 20x20x8 um, 6-12 spheres with
  n in [1.3, 1.6] and kappa in [0, 0.02] (the 3-D volume workload).
* ``disk_stack``     -- a 4-16 layer stack of 64x64 random-disk maps with n in
  [1.0, 1.6] (one instance of the batched sweep).
* ``sweep_instances`` -- the 256-instance sweep: 64 wavelengths in
  [0.4, 0.8] um x 4 incidence angles, orders drawn from {7,11,15,21,25}^2.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


def _pixel_centres(n, period):
    return (np.arange(n) + 0.5) * (period / n)


def triangle_map(seed: int, n: int = 64, period: float = 10.0, n_in: float = 1.4,
                 n_out: float = 1.0) -> np.ndarray:
    """(1, n, n) complex128 map with one seeded triangle (area >= 5 um^2)."""
    rng = np.random.default_rng(seed)
    while True:
        v = rng.uniform(0.0, period, size=(3, 2))
        area = 0.5 * abs((v[1, 0] - v[0, 0]) * (v[2, 1] - v[0, 1]) - (v[2, 0] - v[0, 0]) * (v[1, 1] - v[0, 1]))
        if area >= 5.0:
            break
    c = _pixel_centres(n, period)
    Y, X = np.meshgrid(c, c, indexing="ij")

    def side(a, b):
        return (X - a[0]) * (b[1] - a[1]) - (Y - a[1]) * (b[0] - a[0])

    s0, s1, s2 = side(v[0], v[1]), side(v[1], v[2]), side(v[2], v[0])
    inside = ((s0 >= 0) & (s1 >= 0) & (s2 >= 0)) | ((s0 <= 0) & (s1 <= 0) & (s2 <= 0))
    out = np.full((1, n, n), n_out, dtype=np.complex128)
    out[0][inside] = n_in
    return out


def sphere_volume(seed: int, nxy: int = 128, nz: int = 32, size=(20.0, 20.0, 8.0)) -> np.ndarray:
    """(nz, nxy, nxy) complex128 volume with 6-12 seeded spheres (later ones overwrite)."""
    rng = np.random.default_rng(seed)
    count = int(rng.integers(6, 13))
    cx, cy = _pixel_centres(nxy, size[0]), _pixel_centres(nxy, size[1])
    cz = _pixel_centres(nz, size[2])
    Zg, Yg, Xg = np.meshgrid(cz, cy, cx, indexing="ij")
    vol = np.ones((nz, nxy, nxy), dtype=np.complex128)
    for _ in range(count):
        c = rng.uniform([0, 0, 0], size)
        r = rng.uniform(0.5, 2.0)
        nn = rng.uniform(1.3, 1.6)
        kk = rng.uniform(0.0, 0.02)
        m = (Xg - c[0]) ** 2 + (Yg - c[1]) ** 2 + (Zg - c[2]) ** 2 <= r * r
        vol[m] = complex(nn, kk)
    return vol


def disk_map(rng, n: int = 64, period: float = 25.0) -> np.ndarray:
    """(n, n) complex128 map with 1-8 random disks of n in [1.0, 1.6]."""
    c = _pixel_centres(n, period)
    Y, X = np.meshgrid(c, c, indexing="ij")
    m = np.ones((n, n), dtype=np.complex128)
    for _ in range(int(rng.integers(1, 9))):
        cc = rng.uniform(0, period, 2)
        r = rng.uniform(0.5, 2.5)
        m[(X - cc[0]) ** 2 + (Y - cc[1]) ** 2 <= r * r] = rng.uniform(1.0, 1.6)
    return m


def disk_stack(seed: int, n: int = 64, period: float = 25.0):
    """One sweep instance's stack: (L, n, n) maps and the layer thickness (um).

    scattervolume slices a sample into equal layers (ScatterVolume.cpp:162-168),
    so one thickness in [0.1, 0.5] um is drawn per stack; the slab is L times it.
    """
    rng = np.random.default_rng(seed)
    L = int(rng.integers(4, 17))
    thick = float(rng.uniform(0.1, 0.5))
    maps = np.stack([disk_map(rng, n, period) for _ in range(L)])
    return maps, thick


ORDER_CHOICES = (7, 11, 15, 21, 25)


@dataclass
class SweepInstance:
    """One instance of the batched sweep."""
    index: int
    wavelength: float
    angle_deg: float
    orders: int                 # Mx = My
    maps: np.ndarray            # (L, n, n) complex128
    thickness: float            # layer thickness, um
    period: float

    @property
    def direction(self):
        a = math.radians(self.angle_deg)
        return (math.sin(a), 0.0, math.cos(a))

    @property
    def size(self):
        return (self.period, self.period, self.thickness * self.maps.shape[0])

    def params_kw(self):
        """scattervolume options of this instance (x-polarised, R/T only)."""
        return dict(lambda_=self.wavelength, size=self.size, coef=(self.orders, self.orders),
                    direction=self.direction, ex=(1.0, 0.0), ey=(0.0, 0.0), external=True)


def sweep_instances(seed: int = 0, count: int = 256, n: int = 64, period: float = 25.0):
    """The uneven-instance sweep: 64 wavelengths x 4 angles (x-z plane), seeded."""
    rng = np.random.default_rng(seed)
    nl = max(1, count // 4)
    lams = np.sort(rng.uniform(0.4, 0.8, size=nl))
    angles = (0.0, 10.0, 20.0, 30.0)
    out = []
    for i in range(count):
        lam = float(lams[(i // 4) % nl])
        ang = angles[i % 4]
        m = int(rng.choice(ORDER_CHOICES))
        maps, thick = disk_stack(int(rng.integers(0, 2 ** 31 - 1)), n, period)
        out.append(SweepInstance(i, lam, ang, m, maps, thick, period))
    return out
