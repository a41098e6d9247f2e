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


@pytest.fixture(scope="module")
def cwio_frames(tmp_path_factory):
    """The command-line tools' record-frame code (cli/cwio.hpp) in a small host program."""
    import shutil
    import subprocess
    if shutil.which("g++") is None:
        pytest.skip("no host C++ compiler")
    exe = str(tmp_path_factory.mktemp("cwio") / "cwio_frames")
    root = os.path.dirname(HERE)
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(root, "scattersim_b200", "cli"),
                    os.path.join(HERE, "cwio_frames.cpp"), "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("frame", ["tira", "tira-mirror"])
def test_cli_record_frames_match_the_oracle(fx, cwio_frames, frame, tmp_path):
    """a.cw's fixture records through the CLIs' reader: the Cartesian fields equal the oracle's reading in the
    same frame (own frame, or mirrored for downward waves), and writing them back gives the same bytes."""
    import subprocess
    mirror = frame == "tira-mirror"
    layers = [(float(fx["acw_z"][l]), fx[f"acw_L{l}_Pr_E"], fx[f"acw_L{l}_Pr_k"], fx[f"acw_L{l}_Pt_E"],
               fx[f"acw_L{l}_Pt_k"]) for l in range(3)]
    src, out, fields = (str(tmp_path / n) for n in ("in.cw", "out.cw", "fields.bin"))
    ocw.save(src, fx["acw_Pi_E"], fx["acw_Pi_k"], layers)          # the reference's record pairs, as stored
    r = subprocess.run([cwio_frames, src, frame, out, fields], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(fields, dtype=np.complex128).reshape(-1, 3)
    ref = [ocw.get_e0_tira(fx["acw_Pi_E"], fx["acw_Pi_k"], mirror)]
    for _, PrE, Prk, PtE, Ptk in layers:
        ref += [ocw.get_e0_tira(PrE, Prk, mirror), ocw.get_e0_tira(PtE, Ptk, mirror)]
    ref = np.concatenate(ref)
    assert np.abs(got - ref).max() <= 1e-14 * np.abs(ref).max()
    a, b = open(src, "rb").read(), open(out, "rb").read()
    assert len(a) == len(b)
    E_in, _, lay_in = ocw.load(src)
    E_out, _, lay_out = ocw.load(out)
    assert np.abs(E_out - E_in).max() <= 1e-15 * np.abs(E_in).max()
    for x, y in zip(lay_in, lay_out):
        assert np.abs(y[1] - x[1]).max() <= 1e-15 * np.abs(E_in).max()
        assert np.abs(y[3] - x[3]).max() <= 1e-15 * np.abs(E_in).max()


@pytest.mark.parametrize("run", ["scatterplane", "scatterlayer"])
def test_auto_frame_detection_from_interface_continuity(run, tmp_path):
    """The restated scatterplane / scatterlayer runs written in either convention: the reading that makes the
    field continuous across the first interface is the one the file was written in, so 'auto' recovers it and
    reads the physical fields back."""
    from oracle import scatterlayer as osl
    ks, Es, layers = osl.scatterplane() if run == "scatterplane" else osl.scatterlayer(z=(-3.0, 0.0, 3.0))
    for mirror in (False, True):
        path = str(tmp_path / f"{run}_{int(mirror)}.cw")
        cwfile.save(path, Es, ks, layers, mirror_down=mirror)
        Pi, raw = cwfile._read_raw(path)
        right, wrong = cwfile.interface_jump(Pi, raw, mirror), cwfile.interface_jump(Pi, raw, not mirror)
        assert right < 1e-10 and wrong > 1e-3, (right, wrong)
        assert cwfile.detect_mirror_down(path) == mirror
        E, k, lay = cwfile.load(path, mirror_down="auto")
        scale = np.abs(Es).max()
        assert np.abs(E - Es).max() <= 1e-13 * scale
        # in the mirrored frame a downward wave near 45 degrees (scatterplane's beam about (1, 0, 1)) has a small
        # k'_z = (kx^2 + ky^2 - kz^2) / |k|, and rebuilding the dropped component by k . E = 0 divides by it
        tol = 1e-10 if mirror else 1e-13
        for got, ref in zip(lay, layers):
            for g_, r_ in ((got[1], ref[1]), (got[3], ref[3])):
                assert np.abs(g_ - r_).max() <= tol * max(np.abs(r_).max(), scale)


@pytest.mark.parametrize("rel,mirror", [("data/psf.cw", False), ("x64/a.cw", True)])
def test_auto_frame_detection_on_the_reference_files(cwio_frames, rel, mirror, tmp_path):
    """scatterplane's psf.cw in the own frame, scatterlayer's a.cw in the mirrored one -- by the Python reader
    and by the command-line reader."""
    import subprocess
    ref = os.environ.get("SCATTERSIM_REFERENCE", "")
    path = os.path.join(ref, rel)
    if not ref or not os.path.exists(path):
        pytest.skip("reference tree not mounted")
    assert cwfile.detect_mirror_down(path) == mirror
    fields = str(tmp_path / "f.bin")
    r = subprocess.run([cwio_frames, path, "auto", "-", fields], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    got = np.fromfile(fields, dtype=np.complex128).reshape(-1, 3)
    PiE, Pik, lay = ocw.load(path)
    want = [ocw.get_e0_tira(PiE, Pik, mirror)]
    for _, PrE, Prk, PtE, Ptk in lay:
        want += [ocw.get_e0_tira(PrE, Prk, mirror), ocw.get_e0_tira(PtE, Ptk, mirror)]
    want = np.concatenate(want)
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()


@pytest.mark.parametrize("run", ["scatterplane", "scatterlayer"])
def test_cli_auto_frame_reads_either_convention(cwio_frames, run, tmp_path):
    """The command-line reader's 'auto' frame (cli/cwio.hpp): the restated runs written in either convention
    come back as their Cartesian fields."""
    import subprocess
    from oracle import scatterlayer as osl
    ks, Es, layers = osl.scatterplane() if run == "scatterplane" else osl.scatterlayer(z=(-3.0, 0.0, 3.0))
    ref = np.concatenate([Es] + [a for _, PrE, _, PtE, _ in layers for a in (PrE, PtE)])
    for mirror in (False, True):
        src, fields = str(tmp_path / f"in{int(mirror)}.cw"), str(tmp_path / f"f{int(mirror)}.bin")
        cwfile.save(src, Es, ks, layers, mirror_down=mirror)
        r = subprocess.run([cwio_frames, src, "auto", "-", fields], capture_output=True, text=True)
        assert r.returncode == 0, r.stderr
        got = np.fromfile(fields, dtype=np.complex128).reshape(-1, 3)
        assert np.abs(got - ref).max() <= (1e-10 if mirror else 1e-13) * np.abs(ref).max()
