"""Oracle: ScatterIO files, restated with numpy (test infrastructure only).

ScatterIO.h:18-42 (write_file) and :44-87 (read_file): the plane normal and a
point on the plane as two vec3<double>, then per beam a size_t count N and N
(incident, reflected, transmitted) triples of tira planewave<double> records
(80 bytes: E0x, E0y, kx, ky, kz as complex128).  read_file takes beams until a
count reads as zero (a failed read leaves it zero).  The single-beam and
single-event overloads (:89-117) wrap their arguments in one beam.
"""
from __future__ import annotations

import struct

import numpy as np

RECORD = np.dtype([("E0", "<c16", (2,)), ("k", "<c16", (3,))])   # 80 bytes


def write_file(path, normal, position, incident, reflected, transmitted):
    """incident / reflected / transmitted: lists of beams, each a structured array of RECORD (ScatterIO.h:18-42)."""
    with open(path, "wb") as f:
        f.write(np.asarray(normal, dtype="<f8").tobytes())
        f.write(np.asarray(position, dtype="<f8").tobytes())
        for bi, br, bt in zip(incident, reflected, transmitted):
            f.write(struct.pack("<Q", len(bi)))
            trip = np.empty((len(bi), 3), dtype=RECORD)
            trip[:, 0], trip[:, 1], trip[:, 2] = bi, br, bt
            f.write(trip.tobytes())


def read_file(path):
    """(normal, position, incident, reflected, transmitted) as ScatterIO.h:44-87 reads them."""
    raw = open(path, "rb").read()
    normal = np.frombuffer(raw[0:24], dtype="<f8").copy()
    position = np.frombuffer(raw[24:48], dtype="<f8").copy()
    off = 48
    inc, ref, tra = [], [], []
    while off + 8 <= len(raw):
        (N,) = struct.unpack_from("<Q", raw, off)
        off += 8
        if N == 0:
            break
        trip = np.frombuffer(raw[off:off + N * 3 * RECORD.itemsize], dtype=RECORD).reshape(N, 3)
        off += N * 3 * RECORD.itemsize
        inc.append(trip[:, 0].copy())
        ref.append(trip[:, 1].copy())
        tra.append(trip[:, 2].copy())
    return normal, position, inc, ref, tra
