"""The allocation-free linear solve against the allocating one.

sc_linearsolve_batched_noalloc serves callers that cannot call cudaMalloc:
real-time loops that must not take cudaMalloc's implicit device-wide
synchronisation, and host programs whose framework reserves the GPU's memory
up front and forbids later allocations.  Its scratch is a fixed array in the
library's device memory that every call reuses.  These checks call it through
the C ABI twice in a row -- the second call, on a separate stream, sees the
first call's leftover pivots and status words -- and compare each result with
sc_linearsolve_batched on the same inputs; they also check that a warm call
changes neither the device's free memory nor torch's allocator.  This file is
collected last so a stop-at-first-failure run has already run every other
test.
"""
import ctypes

import numpy as np
import pytest
import torch

from scattersim_b200 import _lib
from scattersim_b200._lib import SC_BADINPUT, SC_OK, SC_SINGULAR

pytestmark = pytest.mark.gpu

TOL = 1e-12   # the two entry points run the same kernels; allow reassociation only


def _colmajor(a):
    return torch.from_numpy(np.ascontiguousarray(np.swapaxes(a, -1, -2))).cuda()


def _noalloc(a, b, n, nrhs, batch, info, stream=None):
    lib = _lib.load()
    sp = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
    return lib.sc_linearsolve_batched_noalloc(ctypes.c_void_p(a.data_ptr()), n, ctypes.c_void_p(b.data_ptr()), nrhs,
                                              batch, info, sp)


def _solve_both(ctx, A, Bm, stream=None):
    lib = _lib.load()
    batch, n, _ = A.shape
    nrhs = Bm.shape[-1]
    a1, b1 = _colmajor(A), _colmajor(Bm)
    a2, b2 = _colmajor(A), _colmajor(Bm)
    info1 = (ctypes.c_int * batch)()
    info2 = (ctypes.c_int * batch)(*([-7] * batch))
    s1 = lib.sc_linearsolve_batched(ctx.handle, ctypes.c_void_p(a1.data_ptr()), n, ctypes.c_void_p(b1.data_ptr()),
                                    nrhs, batch, info1, None)
    torch.cuda.synchronize()
    s2 = _noalloc(a2, b2, n, nrhs, batch, info2, stream)
    x1 = np.swapaxes(b1.cpu().numpy().reshape(batch, nrhs, n), -1, -2)
    x2 = np.swapaxes(b2.cpu().numpy().reshape(batch, nrhs, n), -1, -2)
    return s1, s2, list(info1), list(info2), x1, x2


def test_noalloc_matches_allocating_solve_twice(ctx):
    rng = np.random.default_rng(2024)
    # first call: three regular systems
    A = rng.standard_normal((3, 150, 150)) + 1j * rng.standard_normal((3, 150, 150))
    Bm = rng.standard_normal((3, 150, 4)) + 1j * rng.standard_normal((3, 150, 4))
    s1, s2, i1, i2, x1, x2 = _solve_both(ctx, A, Bm)
    assert s1 == SC_OK and s2 == SC_OK
    assert i1 == i2 == [0, 0, 0]
    assert np.abs(x2 - x1).max() <= TOL * np.abs(x1).max()
    assert np.abs(x2 - np.linalg.solve(A, Bm)).max() <= 1e-10 * np.abs(x1).max()
    # second call, on a separate stream: smaller batch, the second system exactly
    # singular (zero column 5); the leftover pivots and status words of the
    # first call must not leak in
    A = rng.standard_normal((2, 97, 97)) + 1j * rng.standard_normal((2, 97, 97))
    A[1][:, 5] = 0.0
    Bm = rng.standard_normal((2, 97, 3)) + 1j * rng.standard_normal((2, 97, 3))
    s1, s2, i1, i2, x1, x2 = _solve_both(ctx, A, Bm, stream=torch.cuda.Stream())
    assert s1 == SC_SINGULAR and s2 == SC_SINGULAR
    assert i1 == i2 and i1[0] == 0 and i1[1] > 0
    assert np.abs(x2[0] - x1[0]).max() <= TOL * np.abs(x1[0]).max()


def test_noalloc_rejects_sizes_beyond_its_scratch(ctx):
    lib = _lib.load()
    a = torch.zeros(4, dtype=torch.complex128, device="cuda")
    info = (ctypes.c_int * 1)()
    s = lib.sc_linearsolve_batched_noalloc(ctypes.c_void_p(a.data_ptr()), 65537, ctypes.c_void_p(a.data_ptr()), 1,
                                           1, info, None)
    assert s == SC_BADINPUT
    assert b"exceeds the fixed scratch" in lib.sc_last_error_string()
    s = lib.sc_linearsolve_batched_noalloc(ctypes.c_void_p(a.data_ptr()), 2, ctypes.c_void_p(a.data_ptr()), 1,
                                           1025, info, None)
    assert s == SC_BADINPUT


def test_noalloc_allocates_no_device_memory():
    """A warm call leaves the device's free memory and torch's allocator unchanged."""
    rng = np.random.default_rng(7)
    n, batch, nrhs = 120, 4, 2
    A = rng.standard_normal((batch, n, n)) + 1j * rng.standard_normal((batch, n, n))
    Bm = rng.standard_normal((batch, n, nrhs)) + 1j * rng.standard_normal((batch, n, nrhs))
    a, b = _colmajor(A), _colmajor(Bm)
    info = (ctypes.c_int * batch)()
    # a first call loads the kernels (lazy module loading may take device memory once)
    assert _noalloc(a.clone(), b.clone(), n, nrhs, batch, info) == SC_OK
    torch.cuda.synchronize()
    torch_bytes0 = torch.cuda.memory_allocated()
    for _ in range(3):
        a2, b2 = _colmajor(A), _colmajor(Bm)
        torch.cuda.synchronize()
        f_before, _ = torch.cuda.mem_get_info()
        assert _noalloc(a2, b2, n, nrhs, batch, info) == SC_OK
        f_after, _ = torch.cuda.mem_get_info()
        assert f_after == f_before
        assert list(info) == [0] * batch
        del a2, b2
    torch.cuda.synchronize()
    assert torch.cuda.memory_allocated() == torch_bytes0


def test_noalloc_rejects_a_stream_of_another_device():
    """The entry point runs on the current device and refuses another device's stream."""
    if torch.cuda.device_count() < 2:
        pytest.skip("one GPU: no stream of another device to pass")
    a = torch.zeros(4, dtype=torch.complex128, device="cuda:0")
    info = (ctypes.c_int * 1)()
    with torch.cuda.device(1):
        other = torch.cuda.Stream()
    torch.cuda.set_device(0)
    assert _noalloc(a, a, 2, 1, 1, info, other) == SC_BADINPUT


def test_noalloc_records_into_a_cuda_graph():
    """Captured on a side stream into a CUDA graph, after one uncaptured call with the same sizes: the capture
    records the solve without a readback or a synchronisation (info untouched), and each replay, with fresh
    systems copied into the captured buffers, solves them."""
    rng = np.random.default_rng(7)
    batch, n, nrhs = 4, 64, 2

    def systems():
        A = rng.standard_normal((batch, n, n)) + 1j * rng.standard_normal((batch, n, n))
        return A, rng.standard_normal((batch, n, nrhs)) + 1j * rng.standard_normal((batch, n, nrhs))
    A, Bm = systems()
    a, b = _colmajor(A), _colmajor(Bm)
    info = (ctypes.c_int * batch)()
    assert _noalloc(a, b, n, nrhs, batch, info) == SC_OK
    torch.cuda.synchronize()
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    untouched = (ctypes.c_int * batch)(*([-7] * batch))
    with torch.cuda.graph(g, stream=s, capture_error_mode="relaxed"):
        rc = _noalloc(a, b, n, nrhs, batch, untouched, s)
    assert rc == SC_OK and list(untouched) == [-7] * batch
    for _ in range(2):
        A, Bm = systems()
        a.copy_(_colmajor(A))
        b.copy_(_colmajor(Bm))
        g.replay()
        torch.cuda.synchronize()
        x = np.swapaxes(b.cpu().numpy().reshape(batch, nrhs, n), -1, -2)
        assert np.abs(x - np.linalg.solve(A, Bm)).max() <= 1e-10 * np.abs(x).max()
    del g
