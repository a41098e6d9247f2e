"""Generates the golden fixtures in this directory from the reference's shipped data.

    SCATTERSIM_REFERENCE=/path/to/reference python tests/golden/make_golden.py
    python tests/golden/make_golden.py /path/to/reference

Inputs (read-only, from the reference tree):
  data/psf.cw      scatterplane output: 4096 incident waves, one boundary at z=0
  x64/a.cw         scatterlayer output: 4096 incident waves, boundaries -3, 0, 3
  data/layers.npy  the two-slice homogeneous stack of data/generate_layer_volume.py

Outputs:
  cw_fixtures.npz  per file: byte size, sha256, list sizes, boundary z, and every
                   STRIDE-th record of each list (the same incident-wave indices
                   in every list, so each kept wave keeps its reflected and
                   transmitted partners); plus E on a small grid from the full
                   file, evaluated with the oracle's float64 evaluator
  kat_layers.npz   layers.npy, and the oracle's scattervolume (M = 1) and
                   scatterlayer wave amplitudes for it
"""
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import cw as ocw  # noqa: E402
from oracle import scatterlayer as osl  # noqa: E402
from oracle import scattervolume as osv  # noqa: E402

STRIDE = 16


def grid_points(zs):
    """A few points in every region: x-z line through the focus, plus off-axis points."""
    pts = []
    zl = sorted(zs)
    zcand = [zl[0] - 1.0] + [(a + b) / 2 for a, b in zip(zl[:-1], zl[1:])] + [zl[-1] + 1.0] + zl
    for z in zcand:
        for x in (-0.7, 0.0, 0.45):
            pts.append((x, 0.2, z))
    return np.array(pts, dtype=np.float64)


def cw_entry(path, tag, out):
    raw = open(path, "rb").read()
    PiE, Pik, layers = ocw.load(path)
    out[f"{tag}_bytes"] = np.array(len(raw))
    out[f"{tag}_sha256"] = np.frombuffer(hashlib.sha256(raw).digest(), dtype=np.uint8)
    out[f"{tag}_npi"] = np.array(len(PiE))
    out[f"{tag}_z"] = np.array([L[0] for L in layers])
    out[f"{tag}_npr"] = np.array([len(L[1]) for L in layers])
    out[f"{tag}_npt"] = np.array([len(L[3]) for L in layers])
    sel = np.arange(0, len(PiE), STRIDE)
    out[f"{tag}_sel"] = sel
    out[f"{tag}_Pi_E"] = PiE[sel]
    out[f"{tag}_Pi_k"] = Pik[sel]
    for l, (z, PrE, Prk, PtE, Ptk) in enumerate(layers):
        out[f"{tag}_L{l}_Pr_E"] = PrE[sel]
        out[f"{tag}_L{l}_Pr_k"] = Prk[sel]
        out[f"{tag}_L{l}_Pt_E"] = PtE[sel]
        out[f"{tag}_L{l}_Pt_k"] = Ptk[sel]
    # field of the full file, records read in tira's frame as the viewer's getE0() does
    full = [(z, ocw.get_e0_tira(PrE, Prk), Prk, ocw.get_e0_tira(PtE, Ptk), Ptk) for (z, PrE, Prk, PtE, Ptk) in layers]
    zl, b, e, WE, Wk = ocw.unpack(ocw.get_e0_tira(PiE, Pik), Pik, full)
    pts = grid_points(out[f"{tag}_z"])
    out[f"{tag}_pts"] = pts
    out[f"{tag}_E_full"] = ocw.evaluate(pts, zl, b, e, WE, Wk)


def main(ref):
    out = {}
    cw_entry(os.path.join(ref, "data", "psf.cw"), "psf", out)
    cw_entry(os.path.join(ref, "x64", "a.cw"), "acw", out)
    np.savez_compressed(os.path.join(HERE, "cw_fixtures.npz"), **out)

    smp = np.load(os.path.join(ref, "data", "layers.npy"))
    p = osv.Params(lambda_=1.0, n=(1, 1), size=(10, 10, 10), coef=(1, 1))
    sol = osv.solve(smp, p)
    W = osv.build_waves(sol, p)
    inc, waves, ri, z = osl.solve()
    np.savez_compressed(os.path.join(HERE, "kat_layers.npz"), sample=smp, x=sol.x,
                        sv_r_E=W.Pr_E[0], sv_t_E=W.Pt_E[-1], sl_r_E=waves[0][1][0], sl_t_E=waves[-1][2][0],
                        z=np.array(z))
    print("wrote", sorted(out.keys())[:5], "...")


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SCATTERSIM_REFERENCE")
    if not ref:
        sys.exit("usage: make_golden.py REFERENCE_TREE  (or set SCATTERSIM_REFERENCE)")
    main(ref)
