"""CPU model of the modular (Chinese-remainder) int8 GEMM's arithmetic (crt.cu).

Restates with exact integers the steps the kernels take, so that each trick is pinned
without a GPU: operand splitting into 17-bit limbs and the residue with a folded offset
(pack kernels), the accumulator residue with an offset (MMA epilogue), the biased byte
unpacking and the three-limb FP64 reconstruction (rebuild kernel), and a whole emulated
complex product against numpy within the scaling's error bound -- for the engine's 14
moduli and for the first 13 and 12 (smaller P, fewer operand bits), the arithmetic a
count chosen per product would use.
"""
import math

import numpy as np
import pytest

MODS = [255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197]
P = math.prod(MODS)


def sym(v, p):
    r = v % p
    return r - p if r > p // 2 else r


def res_shifted(U, p):
    """(u + h) mod p from U = u + 2^50 split in 17-bit limbs, as the pack kernels form it."""
    U0, U1, U2 = U & 0x1FFFF, (U >> 17) & 0x1FFFF, U >> 34
    c17, c34, c50 = pow(2, 17, p), pow(2, 34, p), pow(2, 50, p)
    v = U2 * c34 + U1 * c17 + U0 + (p - c50) + (p - 1) // 2
    assert 0 <= v < 2 ** 32
    return v % p


def acc_res_shifted(x, p):
    """(x + h) mod p of an int32 accumulator, as the MMA epilogue forms it (unsigned 32-bit wrap)."""
    off = p * ((1 << 31) // p) + (p - 1) // 2
    return ((x + off) & 0xFFFFFFFF) % p


def crt_bits(k, nmod=len(MODS)):
    return min(49, int((math.log2(math.prod(MODS[:nmod])) - 3 - math.log2(2 * max(k, 1))) // 2))


def test_moduli_pairwise_coprime_and_range():
    for i, a in enumerate(MODS):
        assert a % 2 == 1 and a <= 255
        for b in MODS[i + 1:]:
            assert math.gcd(a, b) == 1
    assert 109 < math.log2(P) < 110
    # symmetric residues fit int8
    assert all((p - 1) // 2 <= 127 for p in MODS)


def test_pack_residue_with_folded_offset():
    rng = np.random.default_rng(0)
    us = [int(v) for v in rng.integers(-(2 ** 49), 2 ** 49, 2000)] + [-(2 ** 50) + 1, 2 ** 50 - 1, 0, 1, -1]
    for u in us:
        U = u + 2 ** 50
        for p in MODS:
            h = (p - 1) // 2
            r = res_shifted(U, p) - h          # the kernels subtract h bytewise
            assert r == sym(u, p) and abs(r) <= h
            assert (r & 0xFF) == ((u % p + h) % p - h) & 0xFF


def test_epilogue_accumulator_residue():
    rng = np.random.default_rng(1)
    kmax = (1 << 31) // (128 * 128) - 1          # the host's K' bound: K' 128^2 < 2^31
    lim = kmax * 127 * 127
    xs = [int(v) for v in rng.integers(-lim, lim, 4000)] + [lim, -lim, 0]
    for x in xs:
        for p in MODS:
            assert acc_res_shifted(x, p) - (p - 1) // 2 == sym(x, p)


def test_biased_byte_unpacking():
    for r in range(-128, 128):
        b = r & 0xFF
        assert (b ^ 0x80) == r + 128
    # four residues in a word: byte q of (w ^ 0x80808080), zero-extended, is r_q + 128
    rs = [-127, 0, 5, 127]
    w = sum((r & 0xFF) << (8 * q) for q, r in enumerate(rs))
    for q, r in enumerate(rs):
        assert ((w ^ 0x80808080) >> (8 * q)) & 0xFF == r + 128


def test_biased_byte_packing_every_residue():
    """sym4: bytes r' + (128 - h), XOR 0x80 each, are the int8 bytes of r' - h; sym4_alt: the (a - h, h - c) pairs
    of an A' row 2i, formed by whole-word adds with no carry or borrow between bytes -- all residue pairs, all p."""
    for p in MODS:
        h = (p - 1) // 2
        a, c = np.meshgrid(np.arange(p, dtype=np.int64), np.arange(p, dtype=np.int64), indexing="ij")
        a, c = a.ravel(), c.ravel()
        a1, c1 = np.roll(a, 7), np.roll(c, 3)
        # sym4 on bytes (a, c, a1, c1)
        w = a | (c << 8) | (a1 << 16) | (c1 << 24)
        s = ((w + (128 - h) * 0x01010101) & 0xFFFFFFFF) ^ 0x80808080
        for q, v in enumerate((a, c, a1, c1)):
            byte = (s >> (8 * q)) & 0xFF
            assert np.array_equal(np.where(byte > 127, byte - 256, byte), v - h)
        # sym4_alt
        L = (128 - h) * 0x00010001 + (128 + h) * 0x01000100
        t = (((a + (a1 << 16) + L) - ((c << 8) + (c1 << 24))) & 0xFFFFFFFF) ^ 0x80808080
        for q, v in enumerate((a - h, h - c, a1 - h, h - c1)):
            byte = (t >> (8 * q)) & 0xFF
            assert np.array_equal(np.where(byte > 127, byte - 256, byte), v)


def limbs37(v):
    m = (1 << 37) - 1
    return float(v >> 74), float((v >> 37) & m), float(v & m)


@pytest.mark.parametrize("nmod", [14, 13, 12])
def test_three_limb_reconstruction_is_exact(nmod):
    """S = sum r_p w_p and its reduction by the nearest multiple of P are exact in FP64 limbs -- for the 14
    moduli of the engine and for the first 13 and 12 (a smaller P, fewer residue products)."""
    mods = MODS[:nmod]
    P = math.prod(mods)
    w = []
    for p in mods:
        Mp = P // p
        w.append((Mp * pow(Mp, -1, p)) % P)
    W = [limbs37(v) for v in w]
    PL = limbs37(P)
    rng = np.random.default_rng(2)
    top = (P.bit_length() - 3) - 62                  # |x| up to ~P / 8
    xs = [int(rng.integers(-(2 ** 62), 2 ** 62)) * int(rng.integers(1, 2 ** top)) for _ in range(3000)]
    xs += [0, 1, -1, 2 ** 20 + 7, -(2 ** 60) + 3, 2 ** 75 + 1]       # small values: the absolute error regime
    for x in xs:
        r = [sym(x, p) for p in mods]
        sh = sum(ri * Wi[0] for ri, Wi in zip(r, W))
        sm = sum(ri * Wi[1] for ri, Wi in zip(r, W))
        sl = sum(ri * Wi[2] for ri, Wi in zip(r, W))
        for s_ in (sh, sm, sl):
            assert abs(s_) < 2 ** 52 and s_ == int(s_)   # every partial sum exact in FP64
        s = sh * 2.0 ** 74 + (sm * 2.0 ** 37 + sl)
        q = round(s / P)
        dh, dm, dl = sh - q * PL[0], sm - q * PL[1], sl - q * PL[2]
        for d in (dh, dm, dl):
            assert abs(d) < 2 ** 53 and d == int(d)
        exact = int(dh) * 2 ** 74 + int(dm) * 2 ** 37 + int(dl)
        assert exact == x
        # the kernel's two roundings: fma(dm, 2^37, dl), then fma(dh, 2^74, that) -- the result's own rounding
        # (relative to |x|) plus the inner term's, whose value stays below 2^88 (absolute error < 2^35, far
        # below the operands' rounding: ~2^58 for 14 moduli at k = 1250, ~2^42 and more for 12)
        inner = abs(dm) * 2.0 ** 37 + abs(dl)
        assert inner < 2.0 ** 88
        approx = dh * 2.0 ** 74 + (dm * 2.0 ** 37 + dl)
        assert abs(approx - x) <= 2.0 ** -52 * (abs(x) + inner) + 1.0


@pytest.mark.parametrize("nmod", [14, 13, 12])
@pytest.mark.parametrize("m,n,k", [(1, 1, 1), (7, 5, 9), (24, 17, 33)])
def test_emulated_complex_product(m, n, k, nmod):
    """The whole modular product on small operands: scale rows / columns by powers of two, round to integers
    of `bits` bits, form the interleaved real embedding, multiply residues mod each p exactly, rebuild by CRT
    and scale back -- within the bound the GPU tests state."""
    rng = np.random.default_rng(m * 100 + n * 10 + k)
    A = rng.standard_normal((m, k)) + 1j * rng.standard_normal((m, k))
    B = rng.standard_normal((k, n)) + 1j * rng.standard_normal((k, n))
    A[0] *= 1e-30
    mods = MODS[:nmod]
    P = math.prod(mods)
    bits = crt_bits(k, nmod)
    ea = [math.frexp(max(np.abs(A[i].real).max(), np.abs(A[i].imag).max()))[1] for i in range(m)]
    eb = [math.frexp(max(np.abs(B[:, c].real).max(), np.abs(B[:, c].imag).max()))[1] for c in range(n)]
    ai = [[(int(round(math.ldexp(z.real, bits - ea[i]))), int(round(math.ldexp(z.imag, bits - ea[i]))))
           for z in A[i]] for i in range(m)]
    bi = [[(int(round(math.ldexp(B[j, c].real, bits - eb[c]))), int(round(math.ldexp(B[j, c].imag, bits - eb[c]))))
           for j in range(k)] for c in range(n)]
    C = np.zeros((m, n), complex)
    for i in range(m):
        for c in range(n):
            # rows 2i (Re, -Im) and 2i+1 (Im, Re) of A' against the interleaved column of B'
            re_p, im_p = [], []
            for p in mods:
                sr = si = 0
                for j in range(k):
                    ar, aim = sym(ai[i][j][0], p), sym(ai[i][j][1], p)
                    br, bim = sym(bi[c][j][0], p), sym(bi[c][j][1], p)
                    sr += ar * br - aim * bim
                    si += aim * br + ar * bim
                re_p.append(sym(sr, p))
                im_p.append(sym(si, p))

            def rebuild(res):
                s = sum(r * ((P // p) * pow(P // p, -1, p)) for r, p in zip(res, mods)) % P
                return s - P if s > P // 2 else s
            cr, ci = rebuild(re_p), rebuild(im_p)
            # the exact integer products
            exr = sum(ai[i][j][0] * bi[c][j][0] - ai[i][j][1] * bi[c][j][1] for j in range(k))
            exi = sum(ai[i][j][1] * bi[c][j][0] + ai[i][j][0] * bi[c][j][1] for j in range(k))
            assert (cr, ci) == (exr, exi)
            sc = ea[i] + eb[c] - 2 * bits
            C[i, c] = complex(math.ldexp(cr, sc), math.ldexp(ci, sc))
    ref = A @ B
    ra = np.maximum(np.abs(A.real), np.abs(A.imag)).max(axis=1)
    cb = np.maximum(np.abs(B.real), np.abs(B.imag)).max(axis=0)
    bound = (2.0 * 2.0 ** -bits) * 2 * (2 * ra[:, None]) * (2 * cb[None, :]) * 2 * k + 4e-16 * np.abs(ref)
    assert np.all(np.abs(C - ref) <= bound)
