"""ScatterIO files through the C ABI (host code, no GPU) against the oracle's restatement of ScatterIO.h."""
import ctypes
import os
import tempfile

import numpy as np
import pytest

from oracle import scatterio as osio
from scattersim_b200 import _lib


@pytest.fixture(scope="module")
def lib():
    return _lib.load()


def beams(rng, counts):
    out = []
    for n in counts:
        trips = []
        for _ in range(3):
            r = np.zeros(n, dtype=osio.RECORD)
            r["E0"] = rng.standard_normal((n, 2)) + 1j * rng.standard_normal((n, 2))
            r["k"] = rng.standard_normal((n, 3)) + 1j * rng.standard_normal((n, 3))
            trips.append(r)
        out.append(trips)
    return out


def c_write(lib, path, normal, position, bl):
    counts = (ctypes.c_longlong * max(len(bl), 1))(*[len(b[0]) for b in bl])
    cat = [np.concatenate([b[j] for b in bl]) if bl else np.zeros(0, osio.RECORD) for j in range(3)]
    ptrs = [c.ctypes.data_as(ctypes.c_void_p) for c in cat]
    n = (ctypes.c_double * 3)(*normal)
    p = (ctypes.c_double * 3)(*position)
    return lib.sc_scatterio_write(path.encode(), n, p, len(bl), counts, *ptrs)


def c_read(lib, path):
    n = (ctypes.c_double * 3)()
    p = (ctypes.c_double * 3)()
    nb, ev = ctypes.c_int(0), ctypes.c_longlong(0)
    assert lib.sc_scatterio_read(path.encode(), n, p, ctypes.byref(nb), None, 0, None, None, None, 0,
                                 ctypes.byref(ev)) == _lib.SC_OK
    counts = (ctypes.c_longlong * max(nb.value, 1))()
    recs = [np.zeros(ev.value, dtype=osio.RECORD) for _ in range(3)]
    rc = lib.sc_scatterio_read(path.encode(), n, p, ctypes.byref(nb), counts, nb.value,
                               *[r.ctypes.data_as(ctypes.c_void_p) for r in recs], ev.value, ctypes.byref(ev))
    assert rc == _lib.SC_OK
    return list(n), list(p), list(counts)[:nb.value], recs


def test_c_writer_matches_oracle_bytes_and_reader(lib):
    rng = np.random.default_rng(1)
    bl = beams(rng, [5, 1, 12])
    normal, position = (0.0, 0.0, 1.0), (0.5, -1.5, 3.0)
    with tempfile.TemporaryDirectory() as d:
        a, b = os.path.join(d, "c.sio"), os.path.join(d, "o.sio")
        assert c_write(lib, a, normal, position, bl) == _lib.SC_OK
        osio.write_file(b, normal, position, *[[x[j] for x in bl] for j in range(3)])
        assert open(a, "rb").read() == open(b, "rb").read()
        assert os.path.getsize(a) == 48 + 3 * 8 + 18 * 3 * 80
        nrm, pos, counts, recs = c_read(lib, b)
        assert nrm == list(normal) and pos == list(position) and counts == [5, 1, 12]
        for j in range(3):
            assert np.array_equal(recs[j], np.concatenate([x[j] for x in bl]))
        on, op, oi, orr, ot = osio.read_file(a)
        assert [len(x) for x in oi] == [5, 1, 12]
        assert np.array_equal(np.concatenate(ot), recs[2])


def test_single_event_and_empty_files(lib):
    rng = np.random.default_rng(2)
    bl = beams(rng, [1])
    with tempfile.TemporaryDirectory() as d:
        a = os.path.join(d, "one.sio")
        assert c_write(lib, a, (1, 0, 0), (0, 0, 0), bl) == _lib.SC_OK
        assert c_read(lib, a)[2] == [1]
        e = os.path.join(d, "empty.sio")
        assert c_write(lib, e, (0, 1, 0), (2, 2, 2), []) == _lib.SC_OK
        nrm, pos, counts, recs = c_read(lib, e)
        assert nrm == [0, 1, 0] and pos == [2, 2, 2] and counts == [] and len(recs[0]) == 0


def test_reader_refusals(lib):
    rng = np.random.default_rng(3)
    bl = beams(rng, [4, 4])
    with tempfile.TemporaryDirectory() as d:
        a = os.path.join(d, "t.sio")
        assert c_write(lib, a, (0, 0, 1), (0, 0, 0), bl) == _lib.SC_OK
        raw = open(a, "rb").read()
        cut = os.path.join(d, "cut.sio")
        open(cut, "wb").write(raw[:-40])                 # ends inside the second beam
        n, p = (ctypes.c_double * 3)(), (ctypes.c_double * 3)()
        nb, ev = ctypes.c_int(0), ctypes.c_longlong(0)
        assert lib.sc_scatterio_read(cut.encode(), n, p, ctypes.byref(nb), None, 0, None, None, None, 0,
                                     ctypes.byref(ev)) == _lib.SC_BADINPUT
        small = [np.zeros(3, dtype=osio.RECORD) for _ in range(3)]   # too few slots for 8 events
        counts = (ctypes.c_longlong * 2)()
        assert lib.sc_scatterio_read(a.encode(), n, p, ctypes.byref(nb), counts, 2,
                                     *[r.ctypes.data_as(ctypes.c_void_p) for r in small], 3,
                                     ctypes.byref(ev)) == _lib.SC_BADINPUT
        assert lib.sc_scatterio_read(os.path.join(d, "none.sio").encode(), n, p, ctypes.byref(nb), None, 0,
                                     None, None, None, 0, ctypes.byref(ev)) == _lib.SC_BADINPUT
