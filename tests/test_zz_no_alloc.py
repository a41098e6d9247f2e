"""The allocation-free linear solve against the allocating one.

sc_linearsolve_batched_noalloc serves callers that cannot call cudaMalloc
(solves captured into a CUDA graph, real-time loops, frameworks that forbid
device allocation after start-up); its scratch is a fixed array in the
library's device memory that every call reuses.  These checks call it through
the C ABI twice in a row -- the second call sees the first call's leftover
pivots and status words -- and compare each result with
sc_linearsolve_batched on the same inputs.  This file is collected last so a
stop-at-first-failure run has already run every other test.
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


def _solve_both(ctx, A, Bm):
    lib = _lib.load()
    batch, n, _ = A.shape
    nrhs = Bm.shape[-1]
    a1, b1 = _colmajor(A), _colmajor(Bm)
    a2, b2 = _colmajor(A), _colmajor(Bm)
    info1 = (ctypes.c_int * batch)()
    info2 = (ctypes.c_int * batch)(*([-7] * batch))
    s1 = lib.sc_linearsolve_batched(ctx.handle, ctypes.c_void_p(a1.data_ptr()), n, ctypes.c_void_p(b1.data_ptr()),
                                    nrhs, batch, info1, None)
    s2 = lib.sc_linearsolve_batched_noalloc(ctypes.c_void_p(a2.data_ptr()), n, ctypes.c_void_p(b2.data_ptr()), nrhs,
                                            batch, info2, None)
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
    # second call: smaller batch, the second system exactly singular (zero column 5);
    # the leftover pivots and status words of the first call must not leak in
    A = rng.standard_normal((2, 97, 97)) + 1j * rng.standard_normal((2, 97, 97))
    A[1][:, 5] = 0.0
    Bm = rng.standard_normal((2, 97, 3)) + 1j * rng.standard_normal((2, 97, 3))
    s1, s2, i1, i2, x1, x2 = _solve_both(ctx, A, Bm)
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
