"""The command-line tools' .npy reader and writer (cli/cwio.hpp) against numpy, on the CPU.

The reader takes the sample files of scattervolume --sample (complex128, 2-D or
3-D, C order; the reference loads them with tira's load_npy<complex<double>>,
FourierWave.h:263-278) and refuses what it cannot read with an error; the
writer produces the (N, N, 3) complex64 fields of scattereval (the
scatterview --nogui output, ScatterView.cpp:760-795), which numpy must load.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def tool(tmp_path_factory):
    if shutil.which("g++") is None:
        pytest.skip("no host C++ compiler")
    exe = str(tmp_path_factory.mktemp("npy") / "cwio_npy")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(os.path.dirname(HERE), "scattersim_b200", "cli"),
                    os.path.join(HERE, "cwio_npy.cpp"), "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("shape,dtype,version", [
    ((3, 8, 5), np.complex128, (1, 0)),
    ((8, 5), np.complex128, (1, 0)),
    ((2, 4, 6), np.complex128, (2, 0)),
    ((7, 3), np.float64, (1, 0)),
    ((4, 4, 3), np.complex64, (1, 0)),
])
def test_reader_matches_numpy(tool, tmp_path, shape, dtype, version):
    rng = np.random.default_rng(1)
    a = rng.standard_normal(shape).astype(dtype)
    if np.iscomplexobj(a):
        a = a + 1j * rng.standard_normal(shape).astype(a.real.dtype)
    src, raw = str(tmp_path / "a.npy"), str(tmp_path / "a.bin")
    with open(src, "wb") as f:
        np.lib.format.write_array(f, a, version=version)
    r = subprocess.run([tool, "read", src, raw], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    descr, *dims = r.stdout.split()
    assert descr == a.dtype.str and tuple(int(d) for d in dims) == shape
    assert open(raw, "rb").read() == a.tobytes()


def test_reader_refuses_what_it_cannot_read(tool, tmp_path):
    a = np.ones((4, 5), dtype=np.complex128)
    cases = {
        "fortran.npy": lambda p: np.save(p, np.asfortranarray(a)),
        "bigendian.npy": lambda p: np.save(p, a.astype(">c16")),
        "int.npy": lambda p: np.save(p, np.ones((4, 5), dtype=np.int32)),
    }
    for name, make in cases.items():
        path = str(tmp_path / name)
        make(path)
        r = subprocess.run([tool, "read", path, str(tmp_path / "x.bin")], capture_output=True, text=True)
        assert r.returncode == 1 and "ERROR" in r.stderr, name
    # truncated data and a file that is not .npy
    path = str(tmp_path / "short.npy")
    np.save(path, a)
    data = open(path, "rb").read()
    open(path, "wb").write(data[:-16])
    r = subprocess.run([tool, "read", path, str(tmp_path / "x.bin")], capture_output=True, text=True)
    assert r.returncode == 1 and "truncated" in r.stderr
    open(path, "wb").write(b"not an npy file at all")
    r = subprocess.run([tool, "read", path, str(tmp_path / "x.bin")], capture_output=True, text=True)
    assert r.returncode == 1 and "ERROR" in r.stderr


@pytest.mark.parametrize("shape,dtype", [((16, 16, 3), np.complex64), ((5,), np.float64), ((2, 3, 4), np.complex128)])
def test_writer_output_loads_in_numpy(tool, tmp_path, shape, dtype):
    rng = np.random.default_rng(2)
    a = rng.standard_normal(shape).astype(dtype)
    raw, out = str(tmp_path / "a.bin"), str(tmp_path / "a.npy")
    open(raw, "wb").write(a.tobytes())
    r = subprocess.run([tool, "write", a.dtype.str, raw, out] + [str(s) for s in shape], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr
    b = np.load(out)
    assert b.shape == shape and b.dtype == a.dtype and np.array_equal(a, b)
    header = open(out, "rb").read(10)
    assert header[:8] == b"\x93NUMPY\x01\x00"
    hlen = int.from_bytes(header[8:10], "little")
    assert (10 + hlen) % 64 == 0                     # the data starts on a 64-byte boundary, as numpy writes it
