"""The package's .cw reader/writer (scattersim_b200.cwfile) against the oracle and the reference's files.

Records hold the E0 pair in the frame rotated to Re k; reading rebuilds the
third local component from k . E = 0 -- the reading under which the
reference's shipped files equal the restated solves (tests/test_oracle.py).
"""
import os
import tempfile

import numpy as np
import pytest

from oracle import cw as ocw
from scattersim_b200 import cwfile

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def fx():
    return np.load(os.path.join(HERE, "golden", "cw_fixtures.npz"))


@pytest.mark.parametrize("tag,nl", [("psf", 1), ("acw", 3)])
def test_decode_matches_oracle(fx, tag, nl):
    for key_E, key_k in [(f"{tag}_Pi_E", f"{tag}_Pi_k")] + [(f"{tag}_L{l}_{w}_E", f"{tag}_L{l}_{w}_k")
                                                           for l in range(nl) for w in ("Pr", "Pt")]:
        E2, k = fx[key_E], fx[key_k]
        got = cwfile.from_record(E2, k)
        ref = ocw.get_e0_tira(E2, k)
        assert np.abs(got - ref).max() <= 1e-15 * max(np.abs(ref).max(), 1e-300)
        assert np.abs(cwfile.to_record(got, k) - E2).max() <= 1e-15 * max(np.abs(E2).max(), 1e-300)
        # decoded waves are transverse: k . E = 0
        assert np.abs((got * k).sum(1)).max() <= 1e-13 * np.abs(got).max() * np.abs(k).max()


def test_save_load_roundtrip_and_layout(fx):
    PiE = cwfile.from_record(fx["acw_Pi_E"], fx["acw_Pi_k"])
    layers = []
    for l in range(3):
        layers.append((float(fx["acw_z"][l]), cwfile.from_record(fx[f"acw_L{l}_Pr_E"], fx[f"acw_L{l}_Pr_k"]),
                       fx[f"acw_L{l}_Pr_k"], cwfile.from_record(fx[f"acw_L{l}_Pt_E"], fx[f"acw_L{l}_Pt_k"]),
                       fx[f"acw_L{l}_Pt_k"]))
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "x.cw")
        cwfile.save(path, PiE, fx["acw_Pi_k"], layers)
        n = len(PiE)
        assert os.path.getsize(path) == 16 + 80 * n + 8 + 3 * (8 + 8 + 80 * n + 8 + 80 * n)
        # the oracle's reader sees the reference's record pairs
        E2, k, lay = ocw.load(path)
        assert np.abs(E2 - fx["acw_Pi_E"]).max() <= 1e-15 * np.abs(fx["acw_Pi_E"]).max()
        assert np.array_equal(k, fx["acw_Pi_k"])
        E3, k3, lay3 = cwfile.load(path)
        assert np.abs(E3 - PiE).max() <= 1e-15 * np.abs(PiE).max()
        for a, b in zip(lay3, layers):
            assert a[0] == b[0] and np.abs(a[3] - b[3]).max() <= 1e-15 * max(np.abs(b[3]).max(), 1e-300)


def test_vertical_waves():
    k = np.array([[0, 0, 2.0], [0, 0, -2.0], [0, 0, 2.0 + 0.1j]])
    E = np.array([[1.0, 2.0, 0.0], [1.0, 2.0, 0.0], [0.5j, 1.0, 0.0]])
    assert np.allclose(cwfile.from_record(cwfile.to_record(E, k), k), E)
    assert np.allclose(cwfile.to_record(E, k)[1], [1.0, -2.0])         # half turn about x when going down


@pytest.mark.parametrize("tag,nl", [("psf", 1), ("acw", 3)])
def test_mirrored_decode_matches_oracle(fx, tag, nl):
    """mirror_down reading (downward waves in the frame of their z-mirrored direction) against the oracle's."""
    for l in range(nl):
        for w in ("Pr", "Pt"):
            E2, k = fx[f"{tag}_L{l}_{w}_E"], fx[f"{tag}_L{l}_{w}_k"]
            got = cwfile.from_record(E2, k, mirror_down=True)
            ref = ocw.get_e0_tira(E2, k, mirror_down=True)
            assert np.abs(got - ref).max() <= 1e-15 * max(np.abs(ref).max(), 1e-300)
            assert np.abs(cwfile.to_record(got, k, mirror_down=True) - E2).max() <= 1e-15 * max(np.abs(E2).max(),
                                                                                             1e-300)
            assert np.abs((got * k).sum(1)).max() <= 1e-13 * max(np.abs(got).max(), 1e-300) * np.abs(k).max()
            if w == "Pt":          # upward waves: the same in either reading
                assert np.abs(got - cwfile.from_record(E2, k)).max() <= 1e-15 * max(np.abs(got).max(), 1e-300)


def test_acw_reflected_records_are_the_restated_solve_in_the_mirrored_frame(fx):
    """x64/a.cw's reflected records, read with mirror_down, are the restated scatterlayer solve's Cartesian
    reflected fields; the own-frame reading (right for psf.cw's scatter()-made waves) is not."""
    from oracle import scatterlayer as osl
    _, _, layers = osl.scatterlayer(z=(-3.0, 0.0, 3.0))
    sel = fx["acw_sel"]
    scale = np.abs(fx["acw_Pi_E"]).max()
    for l in range(3):
        PrE = layers[l][1][sel]
        got = cwfile.from_record(fx[f"acw_L{l}_Pr_E"], fx[f"acw_L{l}_Pr_k"], mirror_down=True)
        assert np.abs(got - PrE).max() < 1e-13 * scale
        own = cwfile.from_record(fx[f"acw_L{l}_Pr_E"], fx[f"acw_L{l}_Pr_k"])
        assert np.abs(own - PrE).max() > 1e-2 * scale
