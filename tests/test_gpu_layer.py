"""The batched homogeneous-layer solve and the focused beam on the GPU.

* ``sc_beam_polar`` against the oracle's restatement of SolidAnglePolar
  (pinned by the shipped .cw files), with and without a focal point and an
  obscuration angle;
* ``sc_layer_solve`` against the oracle's per-wave solve of
  ScatterLayer.cpp:110-266 on random stacks of 1 to 15 layers, absorbing and
  not, at oblique beams;
* the scatterplane / scatterlayer default runs against the reference's own
  output files (committed fixture records of data/psf.cw and x64/a.cw), in
  Python and through the command-line tools.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest
import torch

from oracle import cw as ocw
from oracle import scatterlayer as osl
from scattersim_b200 import cwfile, layers, solver

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
BIN = os.path.join(ROOT, "scattersim_b200", "bin")


@pytest.fixture(scope="module")
def ctx():
    c = solver.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def cwfix():
    return np.load(os.path.join(HERE, "golden", "cw_fixtures.npz"))


def _rel(a, b):
    return np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(np.asarray(b)).max(), 1e-300)


@pytest.mark.parametrize("alpha,beta,N,direction,focus", [
    (0.5, 0.0, (64, 64), (1, 0, 1), (0, 0, 0)),        # scatterplane defaults (psf.cw)
    (1.0, 0.0, (64, 64), (0, 0, 1), (0, 0, 0)),        # scatterlayer defaults (a.cw)
    (0.8, 0.2, (17, 9), (0.3, -0.4, 1), (0.5, -1.0, 2.0)),
    (0.0, 0.0, (64, 64), (0.1, 0.2, 1), (1.0, 0.0, 0.0)),   # alpha 0: the centre wave alone
])
def test_beam_matches_oracle(ctx, alpha, beta, N, direction, focus):
    kc, e = osl.incident(0.7, direction, (0.2, 0.1), (1, 0), (0, 0), 1.0)
    ks, Es = layers.beam(ctx, 0.7, kc, e, alpha, beta, N, focus=focus)
    if alpha == 0:
        ok, oE = kc[None, :], e[None, :]
    else:
        ok, oE = osl.beam_polar(alpha, kc, e, N[0], N[1], beta)
    oE = oE * np.exp(-1j * (ok @ np.asarray(focus, dtype=float)))[:, None]
    assert ks.shape[0] == len(ok)
    assert _rel(ks.cpu().numpy(), ok) < 1e-14
    assert _rel(Es.cpu().numpy(), oE) < 1e-13


def _random_stack(rng, L):
    """Incident medium n = 1 (no total internal reflection), thin absorbing layers."""
    n = [1.0] + list(rng.uniform(1.0, 2.2, L - 1))
    kappa = list(np.where(rng.uniform(size=L - 1) < 0.5, rng.uniform(0, 0.1, L - 1), 0.0))
    z = list(np.cumsum(rng.uniform(0.2, 1.0, L - 1)) - 1.5)
    return n, kappa, z


@pytest.mark.parametrize("L,seed", [(1, 0), (2, 1), (3, 2), (4, 3), (7, 4), (11, 5), (15, 6)])
def test_layer_solve_matches_oracle(ctx, L, seed):
    rng = np.random.default_rng(seed)
    n, kappa, z = _random_stack(rng, L)
    lam = float(rng.uniform(0.4, 1.2))
    kc, e = osl.incident(lam, (0.3 * rng.normal(), 0.3 * rng.normal(), 1.0), (1, 0.3), (0.5, 0), (0, 0), n[0])
    ks, Es = layers.beam(ctx, lam, kc, e, 0.6, 0.0, (24, 16))
    rE, rk, tE, tk = layers.layer_solve(ctx, ks, Es, n, kappa, z, lam)
    assert rE.shape == (384, L - 1, 3)
    ks_h, Es_h = ks.cpu().numpy(), Es.cpu().numpy()
    ri = [complex(n[0], 0.0)] + [complex(n[l], kappa[l - 1]) for l in range(1, L)]
    got = [t.cpu().numpy() for t in (rE, rk, tE, tk)]
    scale = np.abs(Es_h).max()
    for w in range(0, 384, 23):
        ref = osl.solve_wave(ks_h[w], Es_h[w], ri, z, 2 * np.pi / lam, n[0])
        for l, (zl, orE, ork, otE, otk) in enumerate(ref):
            assert np.abs(got[0][w, l] - orE).max() < 1e-12 * scale
            assert np.abs(got[2][w, l] - otE).max() < 1e-12 * scale
            assert np.abs(got[1][w, l] - ork).max() < 1e-12 * np.abs(ork).max()
            assert np.abs(got[3][w, l] - otk).max() < 1e-12 * np.abs(otk).max()


def test_layer_solve_energy_lossless(ctx):
    """Lossless stack, x- and y-polarised plane waves: reflected + transmitted z-flux = incident."""
    n, kappa, z = [1.0, 1.7, 1.3, 2.0, 1.5], [0.0, 0.0, 0.0, 0.0], [-1.0, 0.3, 0.9, 2.2]
    lam = 0.63
    for ex, ey in (((1, 0), (0, 0)), ((0, 0), (1, 0))):
        kc, e = osl.incident(lam, (0.4, 0.2, 1.0), ex, ey, (0, 0), n[0])
        ks = torch.tensor(kc[None, :], device="cuda:0")
        Es = torch.tensor(e[None, :], device="cuda:0")
        rE, rk, tE, tk = [t.cpu().numpy()[0] for t in layers.layer_solve(ctx, ks, Es, n, kappa, z, lam)]
        # flux ~ n cos(theta) |E|^2 = Re(kz) |E|^2 / k_vac (non-magnetic media)
        inc = kc[2] * np.vdot(e, e).real
        refl = -rk[0, 2].real * np.vdot(rE[0], rE[0]).real
        trans = tk[-1, 2].real * np.vdot(tE[-1], tE[-1]).real
        assert abs((refl + trans) / inc - 1.0) < 1e-12


def test_scatterplane_reproduces_psf(ctx, cwfix):
    sol = layers.scatterplane(ctx)
    sel = cwfix["psf_sel"]
    k = sol.Pi_k.cpu().numpy()
    E = sol.Pi_E.cpu().numpy()
    scale = np.abs(cwfix["psf_Pi_E"]).max()
    assert np.abs(k[sel] - cwfix["psf_Pi_k"].real).max() < 1e-13
    assert np.abs(cwfile.to_record(E[sel], k[sel]) - cwfix["psf_Pi_E"]).max() < 1e-13 * scale
    rE, rk, tE, tk = (t.cpu().numpy()[:, 0] for t in (sol.Pr_E, sol.Pr_k, sol.Pt_E, sol.Pt_k))
    assert np.abs(rk[sel] - cwfix["psf_L0_Pr_k"]).max() < 1e-13
    assert np.abs(tk[sel] - cwfix["psf_L0_Pt_k"]).max() < 1e-13
    assert np.abs(cwfile.to_record(rE[sel], rk[sel]) - cwfix["psf_L0_Pr_E"]).max() < 1e-13 * scale
    assert np.abs(cwfile.to_record(tE[sel], tk[sel]) - cwfix["psf_L0_Pt_E"]).max() < 1e-13 * scale


def test_scatterlayer_reproduces_acw(ctx, cwfix):
    sol = layers.scatterlayer(ctx, z=(-3.0, 0.0, 3.0))
    sel = cwfix["acw_sel"]
    k = sol.Pi_k.cpu().numpy()
    E = sol.Pi_E.cpu().numpy()
    scale = np.abs(cwfix["acw_Pi_E"]).max()
    assert np.abs(k[sel] - cwfix["acw_Pi_k"].real).max() < 1e-13
    assert np.abs(cwfile.to_record(E[sel], k[sel]) - cwfix["acw_Pi_E"]).max() < 1e-13 * scale
    tE, tk = sol.Pt_E.cpu().numpy(), sol.Pt_k.cpu().numpy()
    rE, rk = sol.Pr_E.cpu().numpy(), sol.Pr_k.cpu().numpy()
    for l in range(3):
        assert np.abs(tk[sel, l] - cwfix[f"acw_L{l}_Pt_k"]).max() < 1e-13
        assert np.abs(cwfile.to_record(tE[sel, l], tk[sel, l]) - cwfix[f"acw_L{l}_Pt_E"]).max() < 1e-13 * scale
        # reflected records: the reference's scatterlayer stores them in the z-mirrored direction's frame
        assert np.abs(rk[sel, l] - cwfix[f"acw_L{l}_Pr_k"]).max() < 1e-13
        assert np.abs(cwfile.to_record(rE[sel, l], rk[sel, l], mirror_down=True) - cwfix[f"acw_L{l}_Pr_E"]).max() \
            < 1e-12 * scale


@pytest.fixture(scope="module")
def tools():
    if not all(os.path.exists(os.path.join(BIN, t)) for t in ("scatterplane", "scatterlayer")):
        subprocess.run(["make", "-C", os.path.join(ROOT, "scattersim_b200", "cli")], check=True)
    return BIN


def _check_file(path, fx, tag, boundaries, check_reflected, reflected_tol=1e-13):
    raw = open(path, "rb").read()
    assert len(raw) == int(fx[f"{tag}_bytes"])          # same list sizes as the reference's file
    PiE, Pik, lay = ocw.load(path)
    sel = fx[f"{tag}_sel"]
    scale = np.abs(fx[f"{tag}_Pi_E"]).max()
    assert np.abs(Pik[sel] - fx[f"{tag}_Pi_k"]).max() < 1e-13
    assert np.abs(PiE[sel] - fx[f"{tag}_Pi_E"]).max() < 1e-13 * scale
    assert [L[0] for L in lay] == list(fx[f"{tag}_z"])
    for l in range(boundaries):
        assert np.abs(lay[l][4][sel] - fx[f"{tag}_L{l}_Pt_k"]).max() < 1e-13
        assert np.abs(lay[l][3][sel] - fx[f"{tag}_L{l}_Pt_E"]).max() < 1e-13 * scale
        assert np.abs(lay[l][2][sel] - fx[f"{tag}_L{l}_Pr_k"]).max() < 1e-13
        if check_reflected:
            assert np.abs(lay[l][1][sel] - fx[f"{tag}_L{l}_Pr_E"]).max() < reflected_tol * scale


def test_cli_scatterplane_writes_psf(tools, cwfix):
    with tempfile.TemporaryDirectory() as d:
        r = subprocess.run([os.path.join(tools, "scatterplane"), "--output", "psf.cw"], cwd=d, capture_output=True,
                           text=True)
        assert r.returncode == 0, r.stderr
        _check_file(os.path.join(d, "psf.cw"), cwfix, "psf", 1, True)


def test_cli_scatterlayer_writes_acw(tools, cwfix):
    with tempfile.TemporaryDirectory() as d:
        r = subprocess.run([os.path.join(tools, "scatterlayer"), "--z", "-3", "0", "3", "--output", "a.cw"], cwd=d,
                           capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        _check_file(os.path.join(d, "a.cw"), cwfix, "acw", 3, False)
        smp = np.load(os.path.join(d, "sample.npy"))
        assert smp.shape == (2, 1, 1) and np.allclose(smp.ravel(), [1.4 + 0.05j, 1.4])


def test_cli_scatterlayer_mirrored_frame_writes_every_acw_record(tools, cwfix):
    """--cw-frame tira-mirror: reflected records in the z-mirrored direction's frame, as the reference's
    scatterlayer stores them -- every record of a.cw, the reflected ones included."""
    with tempfile.TemporaryDirectory() as d:
        r = subprocess.run([os.path.join(tools, "scatterlayer"), "--z", "-3", "0", "3", "--output", "a.cw",
                            "--cw-frame", "tira-mirror"], cwd=d, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        _check_file(os.path.join(d, "a.cw"), cwfix, "acw", 3, True, reflected_tol=1e-12)


def test_cli_layer_tools_reject_bad_input(tools):
    with tempfile.TemporaryDirectory() as d:
        r = subprocess.run([os.path.join(tools, "scatterlayer"), "--mode", "montecarlo"], cwd=d, capture_output=True,
                           text=True)
        assert r.returncode != 0 and "ERROR" in r.stderr
        r = subprocess.run([os.path.join(tools, "scatterplane"), "--n", "1"], cwd=d, capture_output=True, text=True)
        assert r.returncode != 0 and "ERROR" in r.stderr
        r = subprocess.run([os.path.join(tools, "scatterlayer"), "--n"] + ["1.2"] * 16, cwd=d, capture_output=True,
                           text=True)
        assert r.returncode != 0 and "ERROR" in r.stderr
