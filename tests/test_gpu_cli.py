"""The command-line tools end to end: .npy -> scattervolume -> .cw -> scattereval -> .npy.

scattervolume must take the reference's options and write a .cw whose waves
give the oracle's field; scattereval must evaluate a .cw like
`scatterview --nogui` (float32 sum, layer test z >= z_l - 0.001).
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from oracle import cw as ocw
from oracle import scattervolume as osv
from scattersim_b200 import samples

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "scattersim_b200", "bin")


@pytest.fixture(scope="module")
def tools():
    if not os.path.exists(os.path.join(BIN, "scattervolume")):
        subprocess.run(["make", "-C", os.path.join(ROOT, "scattersim_b200", "cli")], check=True)
    return BIN


def test_scattervolume_and_scattereval(tools):
    smp = samples.triangle_map(2)
    kw = dict(lambda_=0.5, size=(10, 10, 1), coef=(5, 5), ex=(1, 0), ey=(0, 0))
    with tempfile.TemporaryDirectory() as d:
        np.save(os.path.join(d, "t.npy"), smp)
        r = subprocess.run([os.path.join(tools, "scattervolume"), "--sample", "t.npy", "--lambda", "0.5",
                            "--size", "10", "10", "1", "--coef", "5", "5", "--ex", "1", "0", "--ey", "0", "0",
                            "--output", "c.cw"], cwd=d, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        assert "Field saved in c.cw." in r.stdout
        assert "Number of Fourier coefficients (Mx, My): [5,5]" in r.stdout
        PiE, Pik, layers = ocw.load(os.path.join(d, "c.cw"))
        # the oracle's wave lists, stored as the reference's records (pair in the frame rotated to Re k)
        p = osv.Params(**kw)
        W = osv.build_waves(osv.solve(smp, p), p)
        assert len(PiE) == 25 and len(layers) == 2
        assert [len(L[1]) for L in layers] == [25, 2 * 25 * 25] and [len(L[3]) for L in layers] == [2 * 25 * 25, 25]
        assert np.allclose(Pik, W.Pi_k) and np.allclose(PiE, ocw.put_e0_tira(W.Pi_E, W.Pi_k))
        assert np.allclose(layers[0][1], ocw.put_e0_tira(W.Pr_E[0], W.Pr_k[0]), atol=1e-12)   # R (wound to z_0)
        assert np.allclose(layers[1][3], ocw.put_e0_tira(W.Pt_E[1], W.Pt_k[1]), atol=1e-12)   # T (wound to z_1)
        # field of the whole file (records read back as getE0() does) vs the oracle's tables
        # through the same store / read round trip (interior modes lose their longitudinal E)
        rt = lambda E, k: ocw.get_e0_tira(ocw.put_e0_tira(E, k), k)
        full = [(z, ocw.get_e0_tira(a, b), b, ocw.get_e0_tira(c, e), e) for (z, a, b, c, e) in layers]
        zl, b, e, WE, Wk = ocw.unpack(ocw.get_e0_tira(PiE, Pik), Pik, full)
        ofull = [(W.z[l], rt(W.Pr_E[l], W.Pr_k[l]), W.Pr_k[l], rt(W.Pt_E[l], W.Pt_k[l]), W.Pt_k[l]) for l in range(2)]
        ozl, ob, oe, oWE, oWk = ocw.unpack(rt(W.Pi_E, W.Pi_k), W.Pi_k, ofull)
        pts = ocw.slice_points(1, (5, 5, 0), 10.0, 32, 5.0)
        Ef = ocw.evaluate(pts, zl, b, e, WE, Wk)
        Eo = ocw.evaluate(pts, ozl, ob, oe, oWE, oWk)
        assert np.linalg.norm(Ef - Eo) / np.linalg.norm(Eo) < 1e-9
        # scattereval: x-z slice at y = 5 through the thin volume
        r = subprocess.run([os.path.join(tools, "scattereval"), "--input", "c.cw", "--nogui", "--size", "10",
                            "--resolution", "5", "--center", "5", "5", "0", "--axis", "1", "--slice", "5",
                            "--output", "xz.npy"], cwd=d, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        E = np.load(os.path.join(d, "xz.npy"))
        assert E.shape == (32, 32, 3) and E.dtype == np.complex64
        # same float32 grid as the tool
        i = np.arange(32, dtype=np.float32)
        dd = np.float32(10.0) / np.float32(31)
        zz, xx = np.meshgrid(np.float32(-5.0) + dd * i, np.float32(0.0) + dd * i, indexing="ij")
        gp = np.stack([xx.ravel(), np.full(1024, np.float32(5.0)), zz.ravel()], -1).astype(np.float64)
        ref = ocw.evaluate(gp, zl.astype(np.float32).astype(np.float64), b, e, WE.astype(np.complex64),
                           Wk.astype(np.complex64), eps=0.001)
        assert np.linalg.norm(E.reshape(-1, 3) - ref) / np.linalg.norm(ref) < 1e-5


def test_scattervolume_rejects_bad_input(tools):
    with tempfile.TemporaryDirectory() as d:
        r = subprocess.run([os.path.join(tools, "scattervolume"), "--sample", "missing.npy"], cwd=d,
                           capture_output=True, text=True)
        assert r.returncode != 0 and "ERROR" in r.stderr
        r = subprocess.run([os.path.join(tools, "scattervolume"), "--bogus", "1"], cwd=d, capture_output=True,
                           text=True)
        assert r.returncode != 0 and "unrecognised option" in r.stderr
