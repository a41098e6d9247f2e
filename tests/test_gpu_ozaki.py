"""The int8 tensor-core complex GEMM (sc_zgemm_emulated_batched) against numpy.

The error bound per element is about (s + 1) 2^-7s x (row scale of A) x
(column scale of B) x k; the tests check it normwise with a margin, plus
exactness on small-integer inputs that the digits represent exactly.
"""
import ctypes

import numpy as np
import pytest
import torch

from scattersim_b200._lib import check

pytestmark = pytest.mark.gpu


def run(ctx, slices, A, B, C=None, alpha=1.0, beta=0.0):
    batch, m, k = A.shape
    n = B.shape[2]
    dA = torch.from_numpy(np.ascontiguousarray(np.swapaxes(A, 1, 2))).cuda()
    dB = torch.from_numpy(np.ascontiguousarray(np.swapaxes(B, 1, 2))).cuda()
    Cin = np.zeros((batch, m, n), complex) if C is None else C
    dC = torch.from_numpy(np.ascontiguousarray(np.swapaxes(Cin, 1, 2))).cuda()
    al = (ctypes.c_double * 2)(complex(alpha).real, complex(alpha).imag)
    be = (ctypes.c_double * 2)(complex(beta).real, complex(beta).imag)
    check(ctx.lib.sc_zgemm_emulated_batched(ctx.handle, slices, m, n, k, al, ctypes.c_void_p(dA.data_ptr()), m, m * k,
                                            ctypes.c_void_p(dB.data_ptr()), k, k * n, be,
                                            ctypes.c_void_p(dC.data_ptr()), m, m * n, batch, None))
    return np.swapaxes(dC.cpu().numpy().reshape(batch, n, m), 1, 2)


def crand(rng, *shape):
    return rng.standard_normal(shape) + 1j * rng.standard_normal(shape)


@pytest.mark.parametrize("m,n,k,batch", [(1, 1, 1, 1), (5, 3, 7, 2), (64, 64, 32, 1), (130, 70, 97, 3),
                                         (300, 129, 260, 2)])
@pytest.mark.parametrize("slices", [3, 7])
def test_emulated_gemm_error_bound(ctx, m, n, k, batch, slices):
    rng = np.random.default_rng(m * 1000 + n + slices)
    A, B, C = crand(rng, batch, m, k), crand(rng, batch, k, n), crand(rng, batch, m, n)
    alpha, beta = 0.7 - 0.2j, -1.1 + 0.4j
    got = run(ctx, slices, A, B, C, alpha, beta)
    ref = alpha * A @ B + beta * C
    # scale of one product term: max row entry x max column entry
    sa = np.abs(np.concatenate([A.real, A.imag], axis=2)).max()
    sb = np.abs(np.concatenate([B.real, B.imag], axis=1)).max()
    bound = (slices + 2) * 2.0 ** (-7 * slices) * 4 * sa * sb * 2 * k * abs(alpha) + 1e-13 * np.abs(ref).max()
    assert np.abs(got - ref).max() <= bound, (np.abs(got - ref).max(), bound)


def test_emulated_gemm_exact_on_small_integers(ctx):
    """Integers below 2^6 in magnitude are one digit under a 2^7 scale: the product is exact."""
    rng = np.random.default_rng(2)
    A = rng.integers(-63, 64, (2, 40, 50)) + 1j * rng.integers(-63, 64, (2, 40, 50))
    B = rng.integers(-63, 64, (2, 50, 30)) + 1j * rng.integers(-63, 64, (2, 50, 30))
    got = run(ctx, 2, A.astype(complex), B.astype(complex))
    assert np.array_equal(got, A @ B)


def test_emulated_gemm_zero_rows_and_scales(ctx):
    """All-zero rows/columns and rows of very different magnitude."""
    rng = np.random.default_rng(3)
    A = crand(rng, 1, 33, 40)
    A[0, 5] = 0
    A[0, 7] *= 1e-200
    A[0, 9] *= 1e150
    B = crand(rng, 1, 40, 17)
    B[0, :, 3] = 0
    got = run(ctx, 7, A, B)
    ref = A @ B
    rowscale = np.abs(A[0]).max(axis=1)[:, None] * np.abs(B[0]).max() * 40
    assert np.all(np.abs(got[0] - ref[0]) <= 1e-13 * rowscale + 1e-300)
    assert np.all(got[0, 5] == 0) and np.all(got[0, :, 3] == 0)
