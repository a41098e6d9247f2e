"""CPU checks of the oracle against the reference's own outputs and invariants.

* The .cw reader/writer reproduces the reference's shipped files byte for
  byte (when the reference tree is mounted) and matches the committed
  fixtures (always).
* The stored E pair of a record is not a Cartesian (E_x, E_y): read that way
  psf.cw jumps at its interface.  It is the pair in tira's frame rotated to
  Re k: read that way psf.cw is continuous, and the restated focused beams
  and layer solves reproduce psf.cw and the incident/transmitted records of
  a.cw to rounding.
* scattervolume at one Fourier order on layers.npy equals the closed-form
  scatterlayer solve (the consistency data/generate_layer_volume.py states).
* Literal-restatement details: fftshift, the column-major reinterpretation,
  the eigen pairing, energy balance.
"""
import hashlib
import os
import tempfile

import numpy as np
import pytest

from oracle import cw as ocw
from oracle import scatterlayer as osl
from oracle import scattervolume as osv
from scattersim_b200 import samples

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
# the reference tree, when mounted (its shipped .cw files); tests that need it skip otherwise
REF = os.environ.get("SCATTERSIM_REFERENCE", "")


@pytest.fixture(scope="module")
def cwfix():
    return np.load(os.path.join(GOLD, "cw_fixtures.npz"))


def _fixture_layers(fx, tag):
    layers = []
    for l in range(len(fx[f"{tag}_z"])):
        layers.append((float(fx[f"{tag}_z"][l]), fx[f"{tag}_L{l}_Pr_E"], fx[f"{tag}_L{l}_Pr_k"],
                       fx[f"{tag}_L{l}_Pt_E"], fx[f"{tag}_L{l}_Pt_k"]))
    return fx[f"{tag}_Pi_E"], fx[f"{tag}_Pi_k"], layers


@pytest.mark.parametrize("tag,rel", [("psf", "data/psf.cw"), ("acw", "x64/a.cw")])
def test_cw_roundtrip_reference_files(cwfix, tag, rel):
    path = os.path.join(REF, rel)
    if not os.path.exists(path):
        pytest.skip("reference tree not mounted")
    raw = open(path, "rb").read()
    assert hashlib.sha256(raw).digest() == bytes(cwfix[f"{tag}_sha256"])
    PiE, Pik, layers = ocw.load(path)
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "x.cw")
        ocw.save(out, PiE, Pik, layers)
        assert open(out, "rb").read() == raw
    sel = cwfix[f"{tag}_sel"]
    assert np.array_equal(PiE[sel], cwfix[f"{tag}_Pi_E"])
    assert np.array_equal(layers[0][1][sel], cwfix[f"{tag}_L0_Pr_E"])


@pytest.mark.parametrize("tag", ["psf", "acw"])
def test_cw_fixture_layout(cwfix, tag):
    """80-byte records: header counts reproduce the shipped file size."""
    npi = int(cwfix[f"{tag}_npi"])
    nrec = npi + int(cwfix[f"{tag}_npr"].sum()) + int(cwfix[f"{tag}_npt"].sum())
    nl = len(cwfix[f"{tag}_z"])
    assert 16 + 80 * nrec + 8 + nl * (8 + 8 + 8) == int(cwfix[f"{tag}_bytes"])


@pytest.mark.parametrize("tag", ["psf", "acw"])
def test_cw_fixture_roundtrip_bytes(cwfix, tag):
    PiE, Pik, layers = _fixture_layers(cwfix, tag)
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "x.cw")
        ocw.save(out, PiE, Pik, layers)
        PiE2, Pik2, layers2 = ocw.load(out)
    assert np.array_equal(PiE2, PiE) and np.array_equal(Pik2, Pik)
    for a, b in zip(layers, layers2):
        assert a[0] == b[0]
        for u, v in zip(a[1:], b[1:]):
            assert np.array_equal(u, v)


def _jump(fx, tag, reader):
    """Largest relative jump of E_x, E_y across the boundaries of a fixture subsample."""
    PiE, Pik, layers = _fixture_layers(fx, tag)
    full = [(z, reader(a, b), b, reader(c, d), d) for (z, a, b, c, d) in layers]
    zl, b, e, WE, Wk = ocw.unpack(reader(PiE, Pik), Pik, full)
    worst = 0.0
    for z in zl:
        pts_a = np.array([[0.3, -0.2, z - 1e-9], [-1.1, 0.4, z - 1e-9], [0.0, 0.0, z - 1e-9]])
        pts_b = pts_a.copy()
        pts_b[:, 2] = z + 1e-9
        Ea = ocw.evaluate(pts_a, zl, b, e, WE, Wk, eps=0.0)
        Eb = ocw.evaluate(pts_b, zl, b, e, WE, Wk, eps=0.0)
        worst = max(worst, np.abs(Ea[:, :2] - Eb[:, :2]).max() / max(np.abs(Ea[:, :2]).max(), 1e-30))
    return worst


def test_cw_records_are_not_cartesian_pairs(cwfix):
    """Read as Cartesian (E0x, E0y) the shipped psf.cw is discontinuous at its interface."""
    assert _jump(cwfix, "psf", ocw.get_e0) > 1e-2


def test_cw_records_in_tira_frame_are_continuous(cwfix):
    """Read in tira's frame (rotated to Re k), psf.cw is continuous across its interface
    (to the phase change over the 2e-9 um between the two evaluation planes)."""
    assert _jump(cwfix, "psf", ocw.get_e0_tira) < 1e-7


def test_tira_frame_roundtrip():
    rng = np.random.default_rng(3)
    k = rng.normal(size=(50, 3)) + 1j * np.concatenate([np.zeros((50, 2)), rng.uniform(0, 0.5, (50, 1))], 1)
    k[:, 2] = np.abs(k[:, 2].real) * np.sign(rng.normal(size=50)) + 1j * k[:, 2].imag
    E = rng.normal(size=(50, 3)) + 1j * rng.normal(size=(50, 3))
    E -= ((E * k).sum(1) / (k * k).sum(1))[:, None] * k          # transverse: k . E = 0
    assert np.allclose(ocw.get_e0_tira(ocw.put_e0_tira(E, k), k), E, atol=1e-12)
    R = ocw.tira_frame(np.array([1.0, 0.0, 1.0]))
    assert np.allclose(R @ R.T, np.eye(3)) and np.allclose(R[:, 2], np.array([1, 0, 1]) / np.sqrt(2))


def _beam_at(fx, tag, ks, Es):
    sel = fx[f"{tag}_sel"]
    return ks[sel], Es[sel]


@pytest.fixture(scope="module")
def psf_restated():
    return osl.scatterplane()


@pytest.fixture(scope="module")
def acw_restated():
    return osl.scatterlayer(z=(-3.0, 0.0, 3.0))


def test_scatterplane_beam_and_solve_reproduce_psf(cwfix, psf_restated):
    """data/psf.cw = scatterplane defaults: polar beam (alpha 0.5, 64 x 64 about (1, 0, 1)),
    one interface n 1 | 1.4 + 0.05i at z = 0; every record agrees to rounding."""
    ks, Es, layers = psf_restated
    sel = cwfix["psf_sel"]
    scale = np.abs(cwfix["psf_Pi_E"]).max()
    assert np.abs(ks[sel] - cwfix["psf_Pi_k"]).max() < 1e-13
    assert np.abs(ocw.put_e0_tira(Es[sel], ks[sel]) - cwfix["psf_Pi_E"]).max() < 1e-13 * scale
    z, PrE, Prk, PtE, Ptk = layers[0]
    assert z == float(cwfix["psf_z"][0])
    assert np.abs(Prk[sel] - cwfix["psf_L0_Pr_k"]).max() < 1e-13
    assert np.abs(Ptk[sel] - cwfix["psf_L0_Pt_k"]).max() < 1e-13
    assert np.abs(ocw.put_e0_tira(PrE[sel], Prk[sel]) - cwfix["psf_L0_Pr_E"]).max() < 1e-13 * scale
    assert np.abs(ocw.put_e0_tira(PtE[sel], Ptk[sel]) - cwfix["psf_L0_Pt_E"]).max() < 1e-13 * scale
    # scatter()-made reflected waves keep their own frame: the mirrored reading is off
    assert np.abs(ocw.put_e0_tira(PrE[sel], Prk[sel], mirror_down=True) - cwfix["psf_L0_Pr_E"]).max() > 1e-2 * scale


def test_scatterlayer_beam_and_solve_reproduce_acw(cwfix, acw_restated):
    """x64/a.cw = scatterlayer's default stack (n 1, 1.4 + 0.05i, 1.4, 1; z -3, 0, 3) under a
    polar beam (alpha 1, 64 x 64 about z): every record agrees to rounding at every boundary.
    The reflected (downward) records, made by tira::planewave's constructor from a Cartesian E0
    (ScatterLayer.cpp:246-251), hold their pair in the frame of the z-mirrored direction; in the
    wave's own frame (the frame of psf.cw's scatter()-made reflected records) they are off."""
    ks, Es, layers = acw_restated
    sel = cwfix["acw_sel"]
    scale = np.abs(cwfix["acw_Pi_E"]).max()
    assert np.abs(ks[sel] - cwfix["acw_Pi_k"]).max() < 1e-13
    assert np.abs(ocw.put_e0_tira(Es[sel], ks[sel]) - cwfix["acw_Pi_E"]).max() < 1e-13 * scale
    for l in range(3):
        z, PrE, Prk, PtE, Ptk = layers[l]
        assert z == float(cwfix["acw_z"][l])
        assert np.abs(Prk[sel] - cwfix[f"acw_L{l}_Pr_k"]).max() < 1e-13
        assert np.abs(Ptk[sel] - cwfix[f"acw_L{l}_Pt_k"]).max() < 1e-13
        assert np.abs(ocw.put_e0_tira(PtE[sel], Ptk[sel]) - cwfix[f"acw_L{l}_Pt_E"]).max() < 1e-13 * scale
        assert np.abs(ocw.put_e0_tira(PrE[sel], Prk[sel], mirror_down=True) - cwfix[f"acw_L{l}_Pr_E"]).max() \
            < 1e-13 * scale
        assert np.abs(ocw.put_e0_tira(PrE[sel], Prk[sel]) - cwfix[f"acw_L{l}_Pr_E"]).max() > 1e-2 * scale
        # upward waves are unaffected by the mirrored reading
        assert np.abs(ocw.put_e0_tira(PtE[sel], Ptk[sel], mirror_down=True) - cwfix[f"acw_L{l}_Pt_E"]).max() \
            < 1e-13 * scale


def test_cw_fixture_field_matches_reference_file(cwfix):
    """The fixture's field values were taken from the full reference file."""
    path = os.path.join(REF, "x64", "a.cw")
    if not os.path.exists(path):
        pytest.skip("reference tree not mounted")
    PiE, Pik, layers = ocw.load(path)
    full = [(z, ocw.get_e0_tira(a, b), b, ocw.get_e0_tira(c, d), d) for (z, a, b, c, d) in layers]
    zl, b, e, WE, Wk = ocw.unpack(ocw.get_e0_tira(PiE, Pik), Pik, full)
    E = ocw.evaluate(cwfix["acw_pts"], zl, b, e, WE, Wk)
    assert np.allclose(E, cwfix["acw_E_full"], rtol=0, atol=1e-12 * np.abs(E).max())


def test_kat_homogeneous_layers():
    kat = np.load(os.path.join(GOLD, "kat_layers.npz"))
    smp = kat["sample"]
    p = osv.Params(lambda_=1.0, n=(1, 1), size=(10, 10, 10), coef=(1, 1))
    sol = osv.solve(smp, p)
    W = osv.build_waves(sol, p)
    inc, waves, ri, z = osl.solve()
    # scattervolume (PI truncated to 3.141592653) vs scatterlayer (M_PI): agree to ~1e-8
    assert np.allclose(W.Pr_E[0][0], waves[0][1][0], atol=1e-7)
    assert np.allclose(W.Pt_E[-1][0], waves[-1][2][0], atol=1e-7)
    assert np.allclose(W.Pr_E[0][0], kat["sv_r_E"][0], atol=1e-13)
    assert np.allclose(waves[-1][2][0], kat["sl_t_E"], atol=1e-13)


@pytest.mark.parametrize("m,n", [(1, 1), (2, 2), (5, 5), (6, 4), (9, 7), (64, 64), (65, 3), (9, 12)])
def test_fftshift_is_matlab_fftshift_for_equal_parity_rows(m, n):
    """fftShift2d takes both shift amounts from the parity of the row count."""
    a = np.arange(m * n, dtype=float).reshape(m, n)
    if m % 2 == 1 or n % 2 == 0:
        assert np.array_equal(osv.fft_shift2d(a), np.fft.fftshift(a))


def test_fftshift_quirk_even_rows_odd_columns():
    """Even x odd: the reference's column table is not a shift (FourierWave.h:97-135)."""
    a = np.arange(2 * 5, dtype=float).reshape(2, 5)
    got = osv.fft_shift2d(a)
    assert not np.array_equal(got, np.fft.fftshift(a))
    assert list(got[1]) == [2.0, 0.0, 1.0, 2.0, 3.0]   # column 4 never appears, column 2 twice


def test_reformat_is_column_major_view():
    data = (np.arange(2 * 3 * 4) + 1j).reshape(2, 3, 4)
    slices, shape = osv.reformat(data)
    assert shape == (2, 3, 4)
    flat = data.reshape(-1)
    for z in range(2):
        for r in range(3):
            for c in range(4):
                assert slices[z][r, c] == flat[z * 12 + r + c * 3]


def test_eigen_sort_pairs_by_imaginary_part():
    lam = np.array([0.5 + 0.2j, -0.5 - 0.2j, 1.0 + 1e-3j, -1.0 - 1e-3j])
    V = np.eye(4, dtype=complex)
    sl, sv = osv.eigen_sort(lam, V)
    assert np.allclose(sl[0::2], [0.5 + 0.2j, 1.0 + 1e-3j])
    assert np.allclose(sl[1::2], [-0.5 - 0.2j, -1.0 - 1e-3j])


@pytest.mark.parametrize("seed,coef,direction", [(0, (5, 5), (0, 0, 1)), (1, (5, 7), (0.3, 0.1, 1))])
def test_energy_balance_lossless(seed, coef, direction):
    smp = samples.triangle_map(seed, n=32)
    p = osv.Params(lambda_=0.5, size=(10, 10, 1), coef=coef, direction=direction)
    sol = osv.solve(smp, p)
    MF = sol.M[0] * sol.M[1]
    x = sol.x
    R = (np.abs(x[0:3 * MF].reshape(3, MF)) ** 2).sum(0) @ sol.Sz0.real
    T = (np.abs(x[3 * MF:].reshape(3, MF)) ** 2).sum(0) @ sol.Sz1.real
    Pin = (np.abs(sol.EF.reshape(3, MF)) ** 2).sum(0) @ sol.Sz0.real
    assert abs((R + T) / Pin - 1.0) < 1e-12


def test_order_clamp_and_pixel_clamp():
    # evanescent clamp fires: 21 orders over a 5 um period at lambda 0.6
    p = osv.Params(lambda_=0.6, size=(5, 5, 1), coef=(21, 21))
    M, msgs = osv.clamp_orders(None, (1, 64, 64), p, np.array([0, 0, 1.0]))
    assert msgs and M[0] < 21 and M[1] < 21
    # pixel clamp: more orders than pixels
    p = osv.Params(lambda_=0.1, size=(10, 10, 1), coef=(31, 31))
    M, msgs = osv.clamp_orders(None, (1, 16, 20), p, np.array([0, 0, 1.0]))
    assert M == [20, 16]
