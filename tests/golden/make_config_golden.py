"""Oracle fixtures at the benchmark workloads' own sizes.

    python tests/golden/make_config_golden.py [thin] [volume] [sweep]

The oracle (oracle/scattervolume.py, numpy/scipy) needs minutes at these
sizes, too long for a test, so its results are committed here and the GPU
tests regenerate the same seeded inputs from scattersim_b200.samples and
compare.  Every fixture stores a checksum of its input so that a change of
the generators is caught instead of compared against.  Each case also stores
the oracle's own sensitivity: the relative change of its output when the
sample is perturbed by 1e-15 relative noise (rounding-level), which bounds
how closely any two correct FP64 implementations can agree.

Outputs (this directory):
  config_thin.npz    the 64x64 seeded triangle map over 10x10 um, lambda 0.5,
                     11x11 orders, x-pol: R/T and the field on every 4th point
                     (both axes) of the 256x256 x-z grid (x in [0, 10],
                     z in [-5, 5], y = 5)
  config_volume.npz  the 128x128x32 seeded sphere volume (seed 1000) over
                     20x20x8 um, lambda 0.6, 10 deg, x-pol, 21x21 orders
                     (1764 x 1764 per layer), all 32 layers: R/T and the field
                     on a 32x32 x-z grid (x in [4, 16], z in [-6, 6], y = 10)
  config_sweep.npz   four instances of the 256-instance sweep (seed 1000) at
                     21x21 and 25x25 orders with their full 12-16 layer stacks,
                     one per incidence angle: R/T
"""
import os
import sys
import time
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import cw as ocw  # noqa: E402
from oracle import scattervolume as osv  # noqa: E402
from scattersim_b200 import samples  # noqa: E402

NOISE = 1e-15
VOLUME_SEED = 1000
SWEEP_SEED = 1000

THIN_KW = dict(lambda_=0.5, size=(10.0, 10.0, 1.0), coef=(11, 11), ex=(1.0, 0.0), ey=(0.0, 0.0))
THIN_GRID = dict(axis=1, center=(5.0, 5.0, 0.0), extent=10.0, N=256, plane=5.0, stride=4)
VOLUME_KW = dict(lambda_=0.6, size=(20.0, 20.0, 8.0), coef=(21, 21),
                 direction=(float(np.sin(np.radians(10.0))), 0.0, float(np.cos(np.radians(10.0)))),
                 ex=(1.0, 0.0), ey=(0.0, 0.0))
VOLUME_GRID = dict(axis=1, center=(10.0, 10.0, 0.0), extent=12.0, N=32, plane=10.0, stride=1)


def checksum(a):
    """crc32 of the array's bytes (C order): identifies the generated input."""
    return np.array(zlib.crc32(np.ascontiguousarray(a).tobytes()), dtype=np.int64)


def grid(g):
    pts = ocw.slice_points(g["axis"], g["center"], g["extent"], g["N"], g["plane"])
    N, s = g["N"], g["stride"]
    keep = (np.arange(N)[:, None] % s == 0) & (np.arange(N)[None, :] % s == 0)
    return pts[keep.ravel()]


def field(sol, p, pts, chunk=8):
    """E at the points from the oracle's wave table, a few points per call (regions hold ~1e6 waves)."""
    W = osv.build_waves(sol, p)
    layers = [(W.z[l], W.Pr_E[l], W.Pr_k[l], W.Pt_E[l], W.Pt_k[l]) for l in range(len(W.z))]
    zl, b, e, WE, Wk = ocw.unpack(W.Pi_E, W.Pi_k, layers)
    out = np.empty((len(pts), 3), dtype=np.complex128)
    for i in range(0, len(pts), chunk):
        out[i:i + chunk] = ocw.evaluate(pts[i:i + chunk], zl, b, e, WE, Wk)
    return out


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def solve_with_sensitivity(smp, kw, pts=None, seed=0):
    p = osv.Params(**kw)
    keep = pts is not None
    sol = osv.solve(smp, p, keep=keep)
    E = field(sol, p, pts) if keep else None
    del sol.eigenvectors[:]
    noisy = smp * (1 + NOISE * np.random.default_rng(seed).standard_normal(smp.shape))
    sol2 = osv.solve(noisy, p, keep=keep)
    sens_x = rel(sol2.x, sol.x)
    sens_E = rel(field(sol2, p, pts), E) if keep else None
    return sol.x, E, sens_x, sens_E


def make_thin():
    smp = samples.triangle_map(0)
    pts = grid(THIN_GRID)
    x, E, sx, sE = solve_with_sensitivity(smp, THIN_KW, pts)
    np.savez_compressed(os.path.join(HERE, "config_thin.npz"), sample_crc=checksum(smp), x=x, pts=pts, E=E,
                        sens_x=sx, sens_E=sE)
    print(f"thin: sensitivity x {sx:.2e} E {sE:.2e}", flush=True)


def make_volume():
    smp = samples.sphere_volume(VOLUME_SEED)
    pts = grid(VOLUME_GRID)
    x, E, sx, sE = solve_with_sensitivity(smp, VOLUME_KW, pts)
    np.savez_compressed(os.path.join(HERE, "config_volume.npz"), sample_crc=checksum(smp), seed=VOLUME_SEED, x=x,
                        pts=pts, E=E, sens_x=sx, sens_E=sE)
    print(f"volume: sensitivity x {sx:.2e} E {sE:.2e}", flush=True)


def pick_sweep_instances(inst):
    """One instance per incidence angle with 21 or 25 orders and >= 12 layers, alternating 21/25."""
    out = []
    for a, want in zip((0.0, 10.0, 20.0, 30.0), (25, 21, 25, 21)):
        cand = [it for it in inst if it.angle_deg == a and it.orders == want and it.maps.shape[0] >= 12]
        if not cand:
            cand = [it for it in inst if it.angle_deg == a and it.orders in (21, 25) and it.maps.shape[0] >= 12]
        out.append(max(cand, key=lambda it: (it.maps.shape[0], it.orders)))
    return out


def make_sweep():
    inst = samples.sweep_instances(SWEEP_SEED, count=256)
    pick = pick_sweep_instances(inst)
    out = {"index": np.array([it.index for it in pick])}
    for j, it in enumerate(pick):
        x, _, sx, _ = solve_with_sensitivity(it.maps, it.params_kw(), seed=j)
        out[f"x{j}"] = x
        out[f"crc{j}"] = checksum(it.maps)
        out[f"sens{j}"] = np.array(sx)
        print(f"sweep instance {it.index}: orders {it.orders} layers {it.maps.shape[0]} angle {it.angle_deg} "
              f"sensitivity {sx:.2e}", flush=True)
    np.savez_compressed(os.path.join(HERE, "config_sweep.npz"), **out)


if __name__ == "__main__":
    which = sys.argv[1:] or ["thin", "sweep", "volume"]
    for w in which:
        t0 = time.time()
        {"thin": make_thin, "volume": make_volume, "sweep": make_sweep}[w]()
        print(f"{w}: {time.time() - t0:.0f} s", flush=True)
