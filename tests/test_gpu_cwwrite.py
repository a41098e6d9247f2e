"""The streaming .cw writer (sc_cw_write) from a device wave table.

Small case: every byte of the structure (size field, counts, z planes, wave
vectors) equals the Python .cw module's file, and the stored E0 pairs agree
with its record-frame rotation to rounding, in every frame (own, Cartesian,
mirrored for downward waves); the file reads
back through the oracle's reader.  Large case: the 3-D volume workload's full
wave table (32 layers, 21x21 orders: about 26 million records, 2 GB) streamed
to disk, its size and sampled records checked.
"""
import ctypes
import os
import struct
import tempfile
import time

import numpy as np
import pytest
import torch

from oracle import cw as ocw
from scattersim_b200 import cwfile, samples, solver
from scattersim_b200._lib import check

pytestmark = pytest.mark.gpu


def list_counts(MF, Z, external):
    interior = 0 if external else 2 * MF * MF
    c = [MF]
    for l in range(Z + 1):
        c += [MF if l == 0 else interior, MF if l == Z else interior]
    return c


def write(ctx, path, wt, counts, frame):
    zl = (ctypes.c_double * len(wt.z_layers))(*wt.z_layers)
    cnt = (ctypes.c_longlong * len(counts))(*counts)
    check(ctx.lib.sc_cw_write(ctx.handle, path.encode(), ctypes.c_void_p(wt.E0.data_ptr()),
                              ctypes.c_void_p(wt.k.data_ptr()), int(wt.E0.shape[0]), len(wt.z_layers), zl, cnt,
                              frame, None))


@pytest.mark.parametrize("external", [False, True])
def test_cw_write_matches_python_writer(ctx, external):
    smp = samples.sphere_volume(5, nxy=24, nz=3, size=(20.0, 20.0, 8.0))
    p = solver.make_params(lambda_=0.6, size=(20, 20, 8), coef=(5, 3), direction=(0.2, 0.1, 0.97), ex=(1, 0),
                           ey=(0, 0.3), external=external)
    sol = solver.solve(ctx, p, torch.from_numpy(smp).cuda())
    wt = solver.waves(ctx, p, sol)
    MF = sol.dims.MF
    counts = list_counts(MF, 3, external)
    E = wt.E0.cpu().numpy()
    K = wt.k.cpu().numpy()
    with tempfile.TemporaryDirectory() as d:
        for frame in (0, 1, 2):
            a = os.path.join(d, f"gpu{frame}.cw")
            write(ctx, a, wt, counts, frame)
            raw = open(a, "rb").read()
            assert len(raw) == 8 + 8 + 8 + 80 * len(E) + len(wt.z_layers) * 24
            # walk the structure: header words exact, records compared
            off = 0
            sz, npi = struct.unpack_from("<QQ", raw, off)
            off += 16
            assert sz == 8 and npi == counts[0]
            recs = [np.frombuffer(raw[off:off + 80 * npi], dtype=np.complex128).reshape(-1, 5)]
            off += 80 * npi
            (nl,) = struct.unpack_from("<Q", raw, off)
            off += 8
            assert nl == len(wt.z_layers)
            for l in range(nl):
                z, npr = struct.unpack_from("<dQ", raw, off)
                off += 16
                assert z == wt.z_layers[l] and npr == counts[1 + 2 * l]
                recs.append(np.frombuffer(raw[off:off + 80 * npr], dtype=np.complex128).reshape(-1, 5))
                off += 80 * npr
                (npt,) = struct.unpack_from("<Q", raw, off)
                off += 8
                assert npt == counts[2 + 2 * l]
                recs.append(np.frombuffer(raw[off:off + 80 * npt], dtype=np.complex128).reshape(-1, 5))
                off += 80 * npt
            assert off == len(raw)
            R = np.concatenate(recs)
            assert np.array_equal(R[:, 2:5], K)                      # wave vectors byte for byte
            pair = E[:, :2] if frame == 1 else cwfile.to_record(E, K, mirror_down=(frame == 2))
            scale = np.abs(E).max(axis=1, keepdims=True) + 1e-300
            assert np.all(np.abs(R[:, 0:2] - pair) <= 4e-16 * scale)
            if frame == 1:
                assert np.array_equal(R[:, 0:2], E[:, :2])
            # the oracle's reader takes the file
            PiE, Pik, layers = ocw.load(a)
            assert len(PiE) == counts[0] and len(layers) == nl


def test_cw_write_volume_workload_size(ctx):
    """The 3-D volume workload's .cw (about 2 GB) streamed from the device table."""
    smp = samples.sphere_volume(1000)
    p = solver.make_params(lambda_=0.6, size=(20.0, 20.0, 8.0), coef=(21, 21),
                           direction=(float(np.sin(np.radians(10.0))), 0.0, float(np.cos(np.radians(10.0)))),
                           ex=(1.0, 0.0), ey=(0.0, 0.0))
    sol = solver.solve(ctx, p, torch.from_numpy(smp).cuda())
    wt = solver.waves(ctx, p, sol)
    nw = int(wt.E0.shape[0])
    counts = list_counts(sol.dims.MF, 32, False)
    assert sum(counts) == nw
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "volume.cw")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        write(ctx, path, wt, counts, 0)
        dt = time.perf_counter() - t0
        size = os.path.getsize(path)
        assert size == 24 + 80 * nw + 33 * 24
        assert size > 1.9e9
        print(f"\n.cw of {nw} records, {size / 1e9:.2f} GB written in {dt:.2f} s ({size / 1e9 / dt:.2f} GB/s)")
        # sampled records: the last transmitted list (file tail) and the start of layer 5's Pt list
        E = wt.E0.cpu().numpy()
        K = wt.k.cpu().numpy()
        with open(path, "rb") as f:
            f.seek(size - 80 * counts[-1])
            tail = np.frombuffer(f.read(80 * counts[-1]), dtype=np.complex128).reshape(-1, 5)
            w0 = sum(counts[:1 + 2 * 5 + 1])          # first wave of Pt_5
            f.seek(24 + 80 * w0 + 24 * 5 + 8 + 8 + 8)
            mid = np.frombuffer(f.read(80 * 64), dtype=np.complex128).reshape(-1, 5)
        assert np.array_equal(tail[:, 2:5], K[-counts[-1]:])
        assert np.allclose(tail[:, 0:2], cwfile.to_record(E[-counts[-1]:], K[-counts[-1]:]), rtol=0,
                           atol=1e-15 * np.abs(E[-counts[-1]:]).max())
        assert np.array_equal(mid[:, 2:5], K[w0:w0 + 64])
