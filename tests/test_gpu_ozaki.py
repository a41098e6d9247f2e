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


# ---------------------------------------------------------------- modular (CRT) engine
def run_crt(ctx, A, B, C=None, alpha=1.0, beta=0.0):
    batch, m, k = A.shape
    n = B.shape[2]
    dA = torch.from_numpy(np.ascontiguousarray(np.swapaxes(A, 1, 2))).cuda()
    dB = torch.from_numpy(np.ascontiguousarray(np.swapaxes(B, 1, 2))).cuda()
    Cin = np.zeros((batch, m, n), complex) if C is None else C
    dC = torch.from_numpy(np.ascontiguousarray(np.swapaxes(Cin, 1, 2))).cuda()
    al = (ctypes.c_double * 2)(complex(alpha).real, complex(alpha).imag)
    be = (ctypes.c_double * 2)(complex(beta).real, complex(beta).imag)
    check(ctx.lib.sc_zgemm_crt_batched(ctx.handle, m, n, k, al, ctypes.c_void_p(dA.data_ptr()), m, m * k,
                                       ctypes.c_void_p(dB.data_ptr()), k, k * n, be,
                                       ctypes.c_void_p(dC.data_ptr()), m, m * n, batch, None))
    return np.swapaxes(dC.cpu().numpy().reshape(batch, n, m), 1, 2)


def crt_bits(k):
    """The engine's scale bits: floor((log2 P - 3 - log2 2k) / 2) with P the product of its 14 moduli."""
    import math
    P = math.prod([255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197])
    return min(49, int((math.log2(P) - 3 - math.log2(2 * max(k, 1))) // 2))


@pytest.mark.parametrize("m,n,k,batch", [(1, 1, 1, 1), (5, 3, 7, 2), (64, 256, 16, 1), (130, 70, 97, 3),
                                         (300, 300, 260, 2), (625, 257, 1250, 1)])
def test_crt_gemm_error_bound(ctx, m, n, k, batch):
    """Rounding each scaled operand to an integer of `bits` bits costs at most 2^-bits of its row / column
    scale; the modular product and the reconstruction are exact, so per element
    |error| <= (2^-bits_A + 2^-bits_B) x 2 x row scale x column scale x 2k (+ FP64 rounding of the result)."""
    rng = np.random.default_rng(m * 1000 + n + 7 * k)
    A, B, C = crand(rng, batch, m, k), crand(rng, batch, k, n), crand(rng, batch, m, n)
    alpha, beta = 0.7 - 0.2j, -1.1 + 0.4j
    got = run_crt(ctx, A, B, C, alpha, beta)
    ref = alpha * A @ B + beta * C
    bits = crt_bits(k)
    ra = np.maximum(np.abs(A.real), np.abs(A.imag)).max(axis=2)          # (batch, m)
    cb = np.maximum(np.abs(B.real), np.abs(B.imag)).max(axis=1)          # (batch, n)
    bound = (2.0 * 2.0 ** -bits) * 2 * (2 * ra[:, :, None]) * (2 * cb[:, None, :]) * 2 * k * abs(alpha)
    bound = bound + 4e-16 * (np.abs(ref) + np.abs(beta * C))
    assert np.all(np.abs(got - ref) <= bound), (np.abs(got - ref) / bound).max()
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-13


def test_crt_gemm_exact_on_integers(ctx):
    """Integer operands below 2^20 are exact after scaling: the product comes back exactly."""
    rng = np.random.default_rng(5)
    A = (rng.integers(-2 ** 19, 2 ** 19, (2, 70, 90)) + 1j * rng.integers(-2 ** 19, 2 ** 19, (2, 70, 90)))
    B = (rng.integers(-2 ** 19, 2 ** 19, (2, 90, 300)) + 1j * rng.integers(-2 ** 19, 2 ** 19, (2, 90, 300)))
    got = run_crt(ctx, A.astype(complex), B.astype(complex))
    assert np.array_equal(got, (A @ B).astype(complex))


def test_crt_gemm_zero_rows_and_scales(ctx):
    """All-zero rows/columns and rows / columns of very different magnitude."""
    rng = np.random.default_rng(6)
    A = crand(rng, 1, 33, 40)
    A[0, 5] = 0
    A[0, 7] *= 1e-200
    A[0, 9] *= 1e150
    B = crand(rng, 1, 40, 17)
    B[0, :, 3] = 0
    B[0, :, 4] *= 1e-100
    got = run_crt(ctx, A, B)
    ref = A @ B
    scale = np.abs(A[0]).max(axis=1)[:, None] * np.abs(B[0]).max(axis=0)[None, :] * 40
    assert np.all(np.abs(got[0] - ref[0]) <= 1e-13 * scale + 1e-300)
    assert np.all(got[0, 5] == 0) and np.all(got[0, :, 3] == 0)


def test_crt_gemm_many_tiles_persistent(ctx):
    """More output tiles than SMs (the persistent CTAs loop over tiles), strided batch, beta = 0."""
    rng = np.random.default_rng(8)
    A, B = crand(rng, 6, 700, 300), crand(rng, 6, 300, 900)
    got = run_crt(ctx, A, B)
    ref = A @ B
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-13


@pytest.mark.parametrize("m,n,k,batch", [(1, 1, 1, 1), (130, 300, 97, 3), (200, 129, 260, 2), (441, 441, 441, 2),
                                         (700, 900, 300, 6)])
def test_crt_pair_tiles_bit_identical(ctx, m, n, k, batch):
    """The CTA-pair kernel (256 x 256 tiles over two SMs) and the single-CTA kernel (128 x 256 tiles) form
    the same exact integer products and the same reconstruction: bit-identical results, including shapes
    whose row tiles are odd in number and whose last column half-tile is all padding."""
    rng = np.random.default_rng(m + 3 * n + 5 * k)
    A, B, C = crand(rng, batch, m, k), crand(rng, batch, k, n), crand(rng, batch, m, n)
    try:
        ctx.crt_tiles(0)
        one = run_crt(ctx, A, B, C, 0.3 + 0.1j, 0.5 - 0.25j)
        ctx.crt_tiles(1)
        two = run_crt(ctx, A, B, C, 0.3 + 0.1j, 0.5 - 0.25j)
    finally:
        ctx.crt_tiles(0)
    assert np.array_equal(one, two)
    ref = (0.3 + 0.1j) * A @ B + (0.5 - 0.25j) * C
    assert np.linalg.norm(two - ref) / np.linalg.norm(ref) < 1e-13
