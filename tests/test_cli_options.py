"""The command-line tools' option surfaces against the reference programs' (no GPU needed).

Help text lists every reference option; unknown options and the inputs the
tools refuse are rejected before any device work, with an ERROR line and a
non-zero exit, as the reference's boost::program_options front ends do.
"""
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "scattersim_b200", "bin")
TOOLS = ("scattervolume", "scattereval", "scatterlayer", "scatterplane")

# option names of ScatterVolume.cpp:511-529, ScatterLayer.cpp:285-303, ScatterPlane.cpp:85-103,
# and the scatterview --nogui slice path (ScatterView.cpp:678-795)
OPTIONS = {
    "scattervolume": ["help", "sample", "lambda", "direction", "ex", "ey", "ez", "n", "kappa", "size", "z", "output",
                      "coef", "psf", "external", "log", "npz"],
    "scattereval": ["input", "size", "resolution", "output", "axis", "center", "slice"],
    "scatterlayer": ["help", "lambda", "direction", "ex", "ey", "ez", "n", "kappa", "z", "output_sample", "output",
                     "alpha", "beta", "na", "samples", "mode"],
    "scatterplane": ["help", "lambda", "direction", "focus", "ex", "ey", "ez", "n", "kappa", "z", "output", "alpha",
                     "beta", "samples", "mode", "wavemask", "nooutput"],
}


@pytest.fixture(scope="module")
def tools():
    if not all(os.path.exists(os.path.join(BIN, t)) for t in TOOLS):
        if not os.path.exists(os.path.join(ROOT, "scattersim_b200", "libscattersim_b200.so")):
            pytest.skip("library not built")
        r = subprocess.run(["make", "-C", os.path.join(ROOT, "scattersim_b200", "cli")], capture_output=True)
        if r.returncode != 0:
            pytest.skip("command-line tools not built")
    return BIN


def _run(tools, tool, *args, cwd=None):
    return subprocess.run([os.path.join(tools, tool), *args], capture_output=True, text=True, cwd=cwd, timeout=60)


@pytest.mark.parametrize("tool", TOOLS)
def test_help_lists_reference_options(tools, tool):
    r = _run(tools, tool, "--help")
    assert r.returncode == 1                           # the reference returns 1 after printing help
    for name in OPTIONS[tool]:
        assert f"--{name}" in r.stdout, name


@pytest.mark.parametrize("tool", TOOLS)
def test_unknown_option_rejected(tools, tool):
    r = _run(tools, tool, "--bogus", "1")
    assert r.returncode != 0 and "unrecognised option" in (r.stderr + r.stdout)


def test_refusals_before_device_work(tools, tmp_path):
    r = _run(tools, "scatterlayer", "--mode", "montecarlo", cwd=tmp_path)
    assert r.returncode != 0 and "ERROR" in r.stderr
    r = _run(tools, "scatterplane", "--n", "1", cwd=tmp_path)
    assert r.returncode != 0 and "ERROR" in r.stderr
    r = _run(tools, "scattervolume", "--lambda", "0.5", cwd=tmp_path)          # no --sample
    assert r.returncode != 0 and "ERROR" in r.stderr
    r = _run(tools, "scattervolume", "--sample", "s.npy", "--cw-frame", "upside-down", cwd=tmp_path)
    assert r.returncode != 0 and "tira-mirror" in r.stderr                   # the error names the choices
    r = _run(tools, "scatterlayer", "--cw-frame", "sideways", cwd=tmp_path)
    assert r.returncode != 0 and "ERROR" in r.stderr
    r = _run(tools, "scattereval", "--axis", "5", cwd=tmp_path)
    assert r.returncode != 0 and "ERROR" in (r.stderr + r.stdout)
    assert not any(tmp_path.iterdir())                  # nothing written
