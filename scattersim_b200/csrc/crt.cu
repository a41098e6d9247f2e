// Complex128 GEMM on the int8 tensor cores by modular arithmetic (the
// Chinese remainder theorem): C_b = alpha * A_b B_b + beta * C_b with about
// 2^-47 relative error per product for K up to ~1300 (fewer bits beyond).
//
// Method (the modular integer emulation published as "Ozaki scheme II",
// Ozaki, Uchino and Imamura, 2025, restated here for complex operands):
//   * Each complex row i of A is scaled by 2^(al - e_i), each column c of B by
//     2^(be - f_c) (e_i, f_c: exponents bounding the row / column), and
//     rounded to integers, |a| <= 2^al, |b| <= 2^be.  The complex product is
//     the real product A' B' of the interleaved embedding used by the
//     digit-sliced engine (rows 2i / 2i+1 of C' are Re / Im of row i), so the
//     exact integer result C'_int = A'_int B'_int satisfies
//     |C'_int| <= 2k 2^(al+be) < P / 4 with P the product of the moduli.
//   * For each of NMOD pairwise coprime moduli p (odd, <= 255) the operands
//     are reduced to symmetric residues (|r| <= 127, int8) and one int8 GEMM
//     on the tensor cores gives A'_p B'_p exactly in int32; its residue mod p
//     is C'_int mod p.
//   * C'_int is rebuilt from its NMOD residues r_p as S = sum_p r_p w_p minus
//     the nearest multiple of P, w_p = (P/p) ((P/p)^-1 mod p) mod P.  The
//     110-bit constants are held as three 37-bit limbs in doubles, so the three
//     limb sums and the reduction by q = round(S / P) are exact in FP64 and
//     only the final limb combination rounds (absolute error ~2^34 on values
//     needing ~2^58).  C = 2^(e_i + f_c - al - be) C'_int.
// NMOD = 14 moduli -> P ~ 2^109.8: al = be = 47 for k <= 1250 (2^-47 per
// element relative to row x column scale x k, on par with 7 digit slices of
// the digit-sliced engine) at 14 int8 products instead of 28.
//
// Data path: pack kernels write, per modulus, the A' and B' residue tiles in
// the UMMA K-major core-matrix layout (as the digit-sliced engine does for its
// digit planes).  The MMA kernel is persistent (one CTA per SM); a CTA owns
// output tiles of 128 rows of C' (64 complex rows) x 256 complex columns and
// for each tile runs NMOD passes of the K loop: warp 0 streams 72 KB stages
// (six K steps: A 24 KB + B 48 KB, two bulk copies) through a 3-slot ring with
// cp.async.bulk, warp 1 issues six 128 x 256 x 32 MMAs per stage (one commit
// per stage: every stage's copy and barrier round trip costs time that the
// MMAs do not hide, so fewer, larger stages run faster: 1, 2, 3, 4, 5, 6 K
// steps per stage measured 2.33, 1.37, 1.12, 0.92, 0.87, 0.85 ms at 1250^3 x 8,
// and 8 steps in two slots 0.90 ms, the ring then too shallow) into one of two
// 256-column TMEM accumulators, and eight epilogue warps turn a finished
// accumulator into int8 residues (in a residue buffer, one plane per modulus)
// while the MMAs of the next modulus run in the other accumulator.  A rebuild
// kernel then reads each output's 14 residues and writes C in FP64.  All
// waits are bounded; a timeout sets the error word and the CTA drains its
// copies, frees its TMEM and returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <mutex>
#include <cstdint>
#include <type_traits>

#include "common.cuh"
#include "kernels.cuh"
#include "tcgen05.cuh"

namespace sc {

namespace {

constexpr int CRT_NMOD = 14;
constexpr int CRT_BM = 128;                  // rows of C' per tile (TMEM lanes)
constexpr int CRT_BN = 256;                  // complex columns per tile
constexpr int CRT_BK = 32;                   // K' bytes per stage
constexpr int CRT_ATILE = CRT_BM * CRT_BK;   // 4 KB
constexpr int CRT_BTILE = CRT_BN * CRT_BK;   // 8 KB
constexpr int CRT_STAGE = CRT_ATILE + CRT_BTILE;   // one K step (the probe's operands)
constexpr int CRT_KSUB = 6;                  // K steps per ring stage: six MMAs per commit
constexpr int CRT_SA = CRT_KSUB * CRT_ATILE;   // 24 KB: the stage's A tiles, consecutive in memory
constexpr int CRT_SB = CRT_KSUB * CRT_BTILE;   // 48 KB
constexpr int CRT_SLOT = CRT_SA + CRT_SB;      // 72 KB
constexpr int CRT_NS = 3;                    // ring slots (216 KB)
constexpr int CRT_EPI_WARPS = 8;
constexpr int CRT_THREADS = 32 * (2 + CRT_EPI_WARPS);
constexpr uint32_t CRT_IDESC = tc::idesc_i8(CRT_BM, CRT_BN);
constexpr int CRT_MODS[CRT_NMOD] = {255, 253, 251, 247, 241, 239, 233, 229, 227, 223, 217, 211, 199, 197};

// moduli, 1/p, the three limbs of w_p and of P, 1/P (filled once per device)
struct CrtConst {
    double p[CRT_NMOD];
    double inv_p[CRT_NMOD];
    double wh[CRT_NMOD], wm[CRT_NMOD], wl[CRT_NMOD];
    double Ph, Pm, Pl, invP;
    double log2P;
};
__constant__ CrtConst c_crt;

// ---------------------------------------------------------------- host constants
// 128-bit unsigned arithmetic for the limbs (P < 2^110)
typedef unsigned __int128 u128;

CrtConst make_constants() {
    CrtConst k{};
    u128 P = 1;
    for (int i = 0; i < CRT_NMOD; ++i) P *= (u128)CRT_MODS[i];
    const u128 mask = ((u128)1 << 37) - 1;
    auto limb = [&](u128 x, double* h, double* m, double* l) {
        *h = (double)(uint64_t)(x >> 74);
        *m = (double)(uint64_t)((x >> 37) & mask);
        *l = (double)(uint64_t)(x & mask);
    };
    for (int i = 0; i < CRT_NMOD; ++i) {
        const uint64_t p = (uint64_t)CRT_MODS[i];
        const u128 Mp = P / p;
        const uint64_t mr = (uint64_t)(Mp % p);
        uint64_t y = 0;   // Mp^-1 mod p by search (p < 256)
        for (uint64_t t = 1; t < p; ++t)
            if ((mr * t) % p == 1) {
                y = t;
                break;
            }
        const u128 w = (Mp * (u128)y) % P;
        k.p[i] = (double)p;
        k.inv_p[i] = 1.0 / (double)p;
        limb(w, &k.wh[i], &k.wm[i], &k.wl[i]);
    }
    limb(P, &k.Ph, &k.Pm, &k.Pl);
    const double Pd = std::ldexp(k.Ph, 74) + std::ldexp(k.Pm, 37) + k.Pl;
    k.invP = 1.0 / Pd;
    k.log2P = std::log2(Pd);
    return k;
}

// scale exponents: al = be = floor((log2 P - 3 - log2 K') / 2), K' = 2k
int crt_bits(int k, double log2P) {
    const double kp = 2.0 * (double)(k > 0 ? k : 1);
    int b = (int)std::floor((log2P - 3.0 - std::log2(kp)) / 2.0);
    return b > 49 ? 49 : b;   // |scaled operand| <= 2^49 < 2^50, the range of the limb split
}

// The residue arithmetic runs in int32 with the moduli as compile-time
// constants (the compiler turns x % p into multiply-high sequences on the
// integer pipes); FP64 rounding and int<->double conversions would all go
// through the conversion (XU) pipe, which then throttles the epilogue.
__host__ __device__ constexpr int crt_mod(int t) {
    return t == 0 ? 255 : t == 1 ? 253 : t == 2 ? 251 : t == 3 ? 247 : t == 4 ? 241 : t == 5 ? 239 : t == 6 ? 233
         : t == 7 ? 229 : t == 8 ? 227 : t == 9 ? 223 : t == 10 ? 217 : t == 11 ? 211 : t == 12 ? 199 : 197;
}
// 2^e mod p for e = 17, 34, 50 (the limb weights of the operand split below)
__host__ __device__ constexpr int pow2_mod(int e, int p) { return e == 0 ? 1 % p : (2 * pow2_mod(e - 1, p)) % p; }

// (x + h) mod p, h = (p - 1) / 2, for an int32 accumulator: |x| <= K' 127^2
// with K' 128^2 < 2^31 (checked on the host), so the offset p floor(2^31 / p)
// + h (= h mod p) keeps x + offset in [0, 2^32) and one unsigned remainder
// gives r' = r + h for the symmetric residue r
template <int P>
__device__ __forceinline__ uint32_t acc_res_shifted(int x) {
    constexpr unsigned OFF = (unsigned)P * ((1u << 31) / (unsigned)P) + (unsigned)(P - 1) / 2;
    return ((unsigned)x + OFF) % (unsigned)P;
}
// x (|x| < 2^50, any double) rounded to the nearest integer and returned as
// the three 17-bit limbs of x + 2^50: 1.5 2^52 + x places the rounded integer
// in the low mantissa bits (no FP64 rounding or conversion instruction)
__device__ __forceinline__ void round_limbs(double x, int& U0, int& U1, int& U2) {
    const double y = x + 6755399441055744.0;                                 // 1.5 * 2^52
    const long long bits = __double_as_longlong(y) & ((1LL << 52) - 1);      // rounded x + 2^51
    const long long U = bits + (1LL << 50) - (1LL << 51);                    // rounded x + 2^50
    U0 = (int)(U & 0x1FFFF);
    U1 = (int)((U >> 17) & 0x1FFFF);
    U2 = (int)(U >> 34);
}

// x * 2^e exactly (a power-of-two multiply when 2^e is a normal double)
__device__ __forceinline__ double scale2(double x, int e) {
    if (e >= -1022 && e <= 1023) return x * __hiloint2double((e + 1023) << 20, 0);
    return ldexp(x, e);
}


// f(std::integral_constant<int, t>) for t = 0 .. NMOD-1 (the modulus a compile-time constant in each call)
template <int T, typename F>
__device__ __forceinline__ void for_each_mod_from(F& f) {
    if constexpr (T < CRT_NMOD) {
        f(std::integral_constant<int, T>());
        for_each_mod_from<T + 1>(f);
    }
}
template <typename F>
__device__ __forceinline__ void for_each_mod(F& f) { for_each_mod_from<0>(f); }
// f(std::integral_constant<int, t>) for one runtime t
template <int T, typename F>
__device__ __forceinline__ void with_mod_from(int t, F& f) {
    if constexpr (T < CRT_NMOD) {
        if (t == T) f(std::integral_constant<int, T>());
        else with_mod_from<T + 1>(t, f);
    }
}
template <typename F>
__device__ __forceinline__ void with_mod(int t, F& f) { with_mod_from<0>(t, f); }

// ---------------------------------------------------------------- packing
// Residues for packing: r' = (u + h) mod p with h = (p - 1) / 2, so that the
// symmetric residue (|r| <= h) is r' - h; u (|u| < 2^50) comes as U = u + 2^50
// in 17-bit limbs, and the constant (p - 2^50 mod p) + h keeps the unsigned
// sum non-negative.  Four such residues go into one word with the bias
// 128 - h added to every byte (128 + h to a byte that carries h - r' for a
// negated residue): each byte then lies in [128 - h, 128 + h], so the word
// adds and subtracts without a carry or borrow between bytes, and XOR 0x80 per
// byte turns r' + 128 - h into the two's-complement byte of r' - h.  Each
// value costs two multiply-adds, an add and the remainder by a constant; each
// word a few integer adds and one XOR.
template <int P>
__device__ __forceinline__ uint32_t res_shifted(int U0, int U1, int U2) {
    constexpr unsigned c17 = pow2_mod(17, P), c34 = pow2_mod(34, P), c50 = pow2_mod(50, P);
    constexpr unsigned K = (unsigned)(P - c50) + (unsigned)(P - 1) / 2;
    const unsigned v = (unsigned)U2 * c34 + (unsigned)U1 * c17 + ((unsigned)U0 + K);
    return v % (unsigned)P;
}
__device__ __forceinline__ uint32_t bytes4(uint32_t b0, uint32_t b1, uint32_t b2, uint32_t b3) {
    return b0 | (b1 << 8) | (b2 << 16) | (b3 << 24);
}
// bytes r'_q (each in [0, p)) -> bytes r'_q - h: bias every byte by 128 - h, then flip its top bit
template <int P>
__device__ __forceinline__ uint32_t sym4(uint32_t packed) {
    return (packed + (uint32_t)(128 - (P - 1) / 2) * 0x01010101u) ^ 0x80808080u;
}
// bytes (a0 - h, h - c0, a1 - h, h - c1) from a_q, c_q in [0, p): even bytes biased by 128 - h, odd
// bytes by 128 + h less c_q
template <int P>
__device__ __forceinline__ uint32_t sym4_alt(uint32_t a0, uint32_t c0, uint32_t a1, uint32_t c1) {
    constexpr uint32_t L = (uint32_t)(128 - (P - 1) / 2) * 0x00010001u + (uint32_t)(128 + (P - 1) / 2) * 0x01000100u;
    return ((a0 + (a1 << 16) + L) - ((c0 << 8) + (c1 << 24))) ^ 0x80808080u;
}

// copy NP planes of `bytes` contiguous bytes each from shared memory to global
// (plane t at dst + t * plane) with 16-byte stores, consecutive threads on
// consecutive addresses
template <int NP>
__device__ __forceinline__ void planes_out(const unsigned char* sm, int bytes, int8_t* dst, long long plane) {
    const int per = bytes / 16;
    for (int e = threadIdx.x; e < NP * per; e += blockDim.x) {
        const int t = e / per, o = (e - t * per) * 16;
        *reinterpret_cast<uint4*>(dst + t * plane + o) = *reinterpret_cast<const uint4*>(sm + t * bytes + o);
    }
}

// A' residue tiles: [b][p][rb][kb][4 KB].  A block packs one tile (64 complex
// rows x 16 complex columns) for all moduli; a thread takes one complex row i
// and 4 complex columns (8 K' bytes) and writes 8 bytes per modulus to each of
// A' rows 2i (Re, -Im pairs) and 2i+1 (Im, Re pairs) in shared memory; the
// block then stores each modulus' 4 KB tile with contiguous 16-byte stores
// (written directly, 8-byte pieces 32 bytes apart left three quarters of each
// written sector empty).  Seven moduli per round (28 KB of shared memory).
__global__ void __launch_bounds__(256) crt_pack_a_kernel(int m, int k, const double2* __restrict__ A,
                                                         const double2* const* Ap, int lda, long long sA,
                                                         const int* __restrict__ rowexp, int al, int RB, int KB,
                                                         int8_t* __restrict__ out) {
    constexpr int HALF = CRT_NMOD / 2;
    __shared__ __align__(16) unsigned char sm[HALF * CRT_ATILE];
    const int b = blockIdx.z;
    const int rb = blockIdx.x, kb = blockIdx.y;
    const double2* a = Ap ? Ap[b] : A + b * sA;
    const int il = threadIdx.x & 63, jq = threadIdx.x >> 6;
    const int i = rb * (CRT_BM / 2) + il, j0 = kb * (CRT_BK / 2) + 4 * jq;
    int lr[4][3], li[4][3];
    const int ex = (i < m) ? rowexp[(long long)b * m + i] : 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        double2 v = make_double2(0.0, 0.0);
        if (i < m && j0 + q < k) v = a[(long long)(j0 + q) * lda + i];
        round_limbs(scale2(v.x, al - ex), lr[q][0], lr[q][1], lr[q][2]);
        round_limbs(scale2(v.y, al - ex), li[q][0], li[q][1], li[q][2]);
    }
    const int o0 = tc::tile_off(2 * il, 8 * jq), o1 = tc::tile_off(2 * il + 1, 8 * jq);
    const long long plane = (long long)RB * KB * CRT_ATILE;
    int8_t* base = out + (long long)b * CRT_NMOD * plane + ((long long)rb * KB + kb) * CRT_ATILE;
    auto one = [&](auto tag) {
        constexpr int T = decltype(tag)::value;
        constexpr int P = crt_mod(T);
        uint32_t dr[4], di[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            dr[q] = res_shifted<P>(lr[q][0], lr[q][1], lr[q][2]);
            di[q] = res_shifted<P>(li[q][0], li[q][1], li[q][2]);
        }
        // row 2i: Re - h, h - Im ; row 2i+1: Im - h, Re - h
        unsigned char* st = sm + (T % HALF) * CRT_ATILE;
        *reinterpret_cast<uint2*>(st + o0) = make_uint2(sym4_alt<P>(dr[0], di[0], dr[1], di[1]),
                                                        sym4_alt<P>(dr[2], di[2], dr[3], di[3]));
        *reinterpret_cast<uint2*>(st + o1) = make_uint2(sym4<P>(bytes4(di[0], dr[0], di[1], dr[1])),
                                                        sym4<P>(bytes4(di[2], dr[2], di[3], dr[3])));
        if constexpr (T % HALF == HALF - 1) {
            __syncthreads();
            planes_out<HALF>(sm, CRT_ATILE, base + (long long)(T - (HALF - 1)) * plane, plane);
            __syncthreads();
        }
    };
    for_each_mod(one);
}

// B' residue tiles (N x K', K-major): [b][p][cb][kb][8 KB] of 256 columns, or
// with `halves` [b][p][2 cb + h][kb][4 KB] of 128 columns (each CTA of a pair
// then loads its half of a 256-column tile as one contiguous run).  A block
// packs 64 columns of a tile (2 KB per modulus, contiguous in either layout);
// a thread takes one column and 4 complex rows (8 bytes of one core-matrix row
// per modulus) into shared memory, and the block stores the 14 runs of 2 KB
// with contiguous 16-byte stores.
__global__ void __launch_bounds__(256) crt_pack_b_kernel(int k, int n, const double2* __restrict__ B,
                                                         const double2* const* Bp, int ldb, long long sB,
                                                         const int* __restrict__ colexp, int be, int CB, int KB,
                                                         int halves, int8_t* __restrict__ out) {
    constexpr int QB = CRT_BTILE / 4;   // 2 KB: 64 columns x 32 K' bytes
    __shared__ __align__(16) unsigned char sm[CRT_NMOD * QB];
    const int b = blockIdx.z;
    const int cb = blockIdx.x >> 2, qt = blockIdx.x & 3, kb = blockIdx.y;
    const double2* bb = Bp ? Bp[b] : B + b * sB;
    const int cq = threadIdx.x & 63, jq = threadIdx.x >> 6;
    const int cl = qt * 64 + cq;
    const int c = cb * CRT_BN + cl, j0 = kb * (CRT_BK / 2) + 4 * jq;
    int lx[8][3];
    const int ex = (c < n) ? colexp[(long long)b * n + c] : 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        double2 v = make_double2(0.0, 0.0);
        if (c < n && j0 + q < k) v = bb[(long long)c * ldb + j0 + q];
        round_limbs(scale2(v.x, be - ex), lx[2 * q][0], lx[2 * q][1], lx[2 * q][2]);
        round_limbs(scale2(v.y, be - ex), lx[2 * q + 1][0], lx[2 * q + 1][1], lx[2 * q + 1][2]);
    }
    // the block's 64 columns are 8 core-matrix row groups: offset cq within its 2 KB run
    const int o = tc::tile_off(cq, 8 * jq);
    const long long plane = (long long)CB * KB * CRT_BTILE;
    int8_t* base = out + (long long)b * CRT_NMOD * plane +
                   (halves ? ((long long)(2 * cb + (qt >> 1)) * KB + kb) * (CRT_BTILE / 2) + (qt & 1) * QB
                           : ((long long)cb * KB + kb) * CRT_BTILE + qt * QB);
    auto one = [&](auto tag) {
        constexpr int T = decltype(tag)::value;
        constexpr int P = crt_mod(T);
        uint32_t d[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) d[q] = res_shifted<P>(lx[q][0], lx[q][1], lx[q][2]);
        *reinterpret_cast<uint2*>(sm + T * QB + o) =
            make_uint2(sym4<P>(bytes4(d[0], d[1], d[2], d[3])), sym4<P>(bytes4(d[4], d[5], d[6], d[7])));
    };
    for_each_mod(one);
    __syncthreads();
    planes_out<CRT_NMOD>(sm, QB, base, plane);
}

// ---------------------------------------------------------------- MMA kernel
struct CrtArgs {
    int m, n, k, RB, CB, KB, batch, ntiles;
    int shift;               // al + be
    const int8_t* Aq;
    const int8_t* Bq;
    const int* rowexp;
    const int* colexp;
    double2 alpha, beta;
    const double2* alphas;
    double2* C;
    double2* const* Cp;
    int ldc;
    long long sC;
    int8_t* res;             // residues: [b][p][Mp rows of C'][Np columns] int8
    int Mp, Np;              // RB x 128, CB x 256
    int* err;
};

// C'_int from its residues (one value), each given as u = r + 128 in [0, 255]:
// exact limb sums, exact reduction, one rounding
__device__ __forceinline__ double crt_value(const uint32_t (&u)[CRT_NMOD]) {
    double sh = 0.0, sm = 0.0, sl = 0.0;
#pragma unroll
    for (int t = 0; t < CRT_NMOD; ++t) {
        // u in the low bits of 2^52: an exact int8 -> double without a conversion instruction
        const double rv = __hiloint2double(0x43300000, (int)u[t]) - 4503599627370624.0;   // 2^52 + 128
        sh = fma(rv, c_crt.wh[t], sh);
        sm = fma(rv, c_crt.wm[t], sm);
        sl = fma(rv, c_crt.wl[t], sl);
    }
    const double s = fma(sh, 0x1p74, fma(sm, 0x1p37, sl));
    const double q = (s * c_crt.invP + 6755399441055744.0) - 6755399441055744.0;     // round to nearest
    const double dh = fma(-q, c_crt.Ph, sh);
    const double dm = fma(-q, c_crt.Pm, sm);
    const double dl = fma(-q, c_crt.Pl, sl);
    return fma(dh, 0x1p74, fma(dm, 0x1p37, dl));
}

// One CTA's epilogue for one output tile: 128 rows of C' (its TMEM lanes; warp
// w reads lane quarter w % 4, and the two warps of a quarter split the 256
// columns).  For each modulus pass: wait for the accumulator, reduce it to
// int8 residues in the residue buffer and hand the accumulator back.  rb is
// the 128-row tile, cb the 256-column tile; u counts accumulator uses.
// Returns false when a wait gave up (the error word is then set).  The FP64
// rebuild of C from the residues is crt_rebuild_kernel's: done here it kept
// the epilogue warps from draining the next tile's accumulators and stalled
// the MMAs for about a third of the kernel.
template <typename WaitFull, typename Release>
__device__ __forceinline__ bool crt_extract_tile(const CrtArgs& g, uint32_t tmem, int rb, int cb, int b, long long& u,
                                                 volatile int* aborted, WaitFull wait_full, Release release) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ew = warp - 2;
    const int quarter = warp & 3;
    const int half = ew >> 2;
    const int row = quarter * 32 + lane;                 // row of C' in the tile
    for (int t = 0; t < CRT_NMOD; ++t, ++u) {
        const int buf = (int)(u & 1);
        bool ready = !*aborted && wait_full(buf, (uint32_t)((u >> 1) & 1));
        ready = __all_sync(0xffffffffu, ready);
        if (!ready) {
            if (lane == 0 && !*aborted) atomicExch(g.err, 14);
            return false;
        }
        tc::fence_after_sync();
        int8_t* dst = g.res + (((long long)b * CRT_NMOD + t) * g.Mp + (long long)rb * CRT_BM + row) * g.Np +
                      (long long)cb * CRT_BN;
        auto extract = [&](auto tag) {
            constexpr int P = crt_mod(decltype(tag)::value);
#pragma unroll 1
            for (int c0 = half * 128; c0 < half * 128 + 128; c0 += 32) {
                uint32_t r[32];
                tc::tmem_ld32(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(buf * CRT_BN + c0), r);
                uint32_t w[8];
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    w[q] = sym4<P>(bytes4(acc_res_shifted<P>((int)r[4 * q]), acc_res_shifted<P>((int)r[4 * q + 1]),
                                          acc_res_shifted<P>((int)r[4 * q + 2]), acc_res_shifted<P>((int)r[4 * q + 3])));
                *reinterpret_cast<uint4*>(dst + c0) = make_uint4(w[0], w[1], w[2], w[3]);
                *reinterpret_cast<uint4*>(dst + c0 + 16) = make_uint4(w[4], w[5], w[6], w[7]);
            }
        };
        with_mod(t, extract);
        tc::fence_before_sync();
        __syncwarp();
        if (lane == 0) release(buf);
    }
    return true;
}

// C = alpha 2^(e_i + f_c - al - be) C'_int + beta C from the residues: block of
// 8 warps = 8 complex rows i (C' rows 2i, 2i+1) x 256 columns, a lane 8
// consecutive columns (8-byte residue loads, coalesced along the rows).  The
// values go through shared memory so that the stores to the column-major C
// are whole: a quarter-warp writes the block's 8 rows of one column (128
// contiguous bytes).  Tile [256 columns][8 rows] of double2, the row slot
// XOR-swizzled by column / 8 so that neither pass has bank conflicts.
__global__ void __launch_bounds__(256) crt_rebuild_kernel(CrtArgs g) {
    __shared__ double2 tile[256 * 8];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int b = blockIdx.z;
    const int i0 = blockIdx.y * 8, cb0 = blockIdx.x * 256;
    const int i = i0 + warp;
    const int c0 = cb0 + 8 * lane;
    double2* C = g.Cp ? g.Cp[b] : g.C + b * g.sC;
    const double2 alpha = g.alphas ? cmul(g.alpha, g.alphas[b]) : g.alpha;
    const bool beta_zero = (g.beta.x == 0.0 && g.beta.y == 0.0);
    if (i < g.m && c0 < g.n) {
        const long long plane = (long long)g.Mp * g.Np;
        const int8_t* base = g.res + (long long)b * CRT_NMOD * plane + (long long)(2 * i) * g.Np + c0;
        uint2 re[CRT_NMOD], im[CRT_NMOD];
#pragma unroll
        for (int t = 0; t < CRT_NMOD; ++t) {
            re[t] = *reinterpret_cast<const uint2*>(base + t * plane);
            im[t] = *reinterpret_cast<const uint2*>(base + t * plane + g.Np);
        }
        const int ex = g.rowexp[(long long)b * g.m + i] - g.shift;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            const int c = c0 + q;
            if (c >= g.n) break;
            uint32_t rr[CRT_NMOD], ri[CRT_NMOD];
#pragma unroll
            for (int t = 0; t < CRT_NMOD; ++t) {
                // the residue byte r (two's complement) plus 128 is the byte XOR 0x80, zero-extended
                const uint32_t wr = ((q < 4) ? re[t].x : re[t].y) ^ 0x80808080u;
                const uint32_t wi = ((q < 4) ? im[t].x : im[t].y) ^ 0x80808080u;
                rr[t] = __byte_perm(wr, 0u, 0x4440u | (uint32_t)(q & 3));
                ri[t] = __byte_perm(wi, 0u, 0x4440u | (uint32_t)(q & 3));
            }
            const int e = ex + g.colexp[(long long)b * g.n + c];
            const int cl = 8 * lane + q;
            tile[cl * 8 + (warp ^ (lane & 7))] = cmul(alpha, make_double2(scale2(crt_value(rr), e),
                                                                          scale2(crt_value(ri), e)));
        }
    }
    __syncthreads();
    // quarter-warp per column: lanes 8j..8j+7 write rows i0..i0+7 of column 4 it + j (of this warp's 32)
    const int r = lane & 7;
#pragma unroll 4
    for (int it = 0; it < 8; ++it) {
        const int cl = warp * 32 + 4 * it + (lane >> 3);
        const int c = cb0 + cl, row = i0 + r;
        if (c < g.n && row < g.m) {
            double2 val = tile[cl * 8 + (r ^ ((cl >> 3) & 7))];
            double2* pc = C + (long long)c * g.ldc + row;
            if (!beta_zero) val = cfma(g.beta, *pc, val);
            *pc = val;
        }
    }
}

__global__ void __launch_bounds__(CRT_THREADS, 1) crt_mma_kernel(CrtArgs g) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[CRT_NS], empty[CRT_NS], accfull[2], accempty[2];
    __shared__ uint32_t tmem_base;
    __shared__ int abort_flag;
    volatile int* aborted = &abort_flag;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int KB = g.KB;

    if (threadIdx.x == 0) {
        for (int q = 0; q < CRT_NS; ++q) {
            tc::mbar_init(&full[q], 1);
            tc::mbar_init(&empty[q], 1);
        }
        for (int q = 0; q < 2; ++q) {
            tc::mbar_init(&accfull[q], 1);
            tc::mbar_init(&accempty[q], CRT_EPI_WARPS);
        }
        *aborted = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) tc::tmem_alloc(&tmem_base, 512u);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_base;
    const long long planeA = (long long)g.RB * KB * CRT_ATILE;
    const long long planeB = (long long)g.CB * KB * CRT_BTILE;

    if (warp == 0) {
        if (lane == 0) {
            // producer: for each tile, modulus and K step, one A and one B tile
            long long stage = 0;
            for (int tile = blockIdx.x; tile < g.ntiles && !*aborted; tile += gridDim.x) {
                const int cb = tile % g.CB, rb = (tile / g.CB) % g.RB, b = tile / (g.CB * g.RB);
                for (int t = 0; t < CRT_NMOD && !*aborted; ++t) {
                    const int8_t* Ab = g.Aq + ((long long)b * CRT_NMOD + t) * planeA + (long long)rb * KB * CRT_ATILE;
                    const int8_t* Bb = g.Bq + ((long long)b * CRT_NMOD + t) * planeB + (long long)cb * KB * CRT_BTILE;
                    for (int kb = 0; kb < KB; kb += CRT_KSUB, ++stage) {
                        const int nsub = min(CRT_KSUB, KB - kb);
                        const int slot = (int)(stage % CRT_NS);
                        if (stage >= CRT_NS && !tc::mbar_wait(&empty[slot], (uint32_t)(((stage / CRT_NS) - 1) & 1))) {
                            atomicExch(g.err, 11);
                            *aborted = 1;
                            break;
                        }
                        if (*aborted) break;
                        unsigned char* sa = smem_raw + (size_t)slot * CRT_SLOT;
                        tc::mbar_expect_tx(&full[slot], (uint32_t)(nsub * CRT_STAGE));
                        tc::bulk_g2s(sa, Ab + (long long)kb * CRT_ATILE, (uint32_t)(nsub * CRT_ATILE), &full[slot]);
                        tc::bulk_g2s(sa + CRT_SA, Bb + (long long)kb * CRT_BTILE, (uint32_t)(nsub * CRT_BTILE),
                                     &full[slot]);
                    }
                }
            }
            // drain: the last CRT_NS stages' copies must have landed before the CTA exits
            for (long long s2 = (stage > CRT_NS ? stage - CRT_NS : 0); s2 < stage; ++s2)
                tc::mbar_wait(&full[s2 % CRT_NS], (uint32_t)((s2 / CRT_NS) & 1));
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // MMA issuer: accumulator unit u (tile, modulus) in buffer u & 1
            const uint64_t desc0 = tc::smem_desc(smem_raw);
            const uint64_t slot_step = (uint64_t)(CRT_SLOT >> 4);
            long long stage = 0, u = 0;
            for (int tile = blockIdx.x; tile < g.ntiles && !*aborted; tile += gridDim.x) {
                for (int t = 0; t < CRT_NMOD && !*aborted; ++t, ++u) {
                    const int buf = (int)(u & 1);
                    if (u >= 2 && !tc::mbar_wait(&accempty[buf], (uint32_t)(((u >> 1) - 1) & 1))) {
                        atomicExch(g.err, 12);
                        *aborted = 1;
                        break;
                    }
                    tc::fence_after_sync();
                    const uint32_t acc = tmem + (uint32_t)(buf * CRT_BN);
                    for (int kb = 0; kb < KB; kb += CRT_KSUB, ++stage) {
                        const int nsub = min(CRT_KSUB, KB - kb);
                        const int slot = (int)(stage % CRT_NS);
                        if (!tc::mbar_wait(&full[slot], (uint32_t)((stage / CRT_NS) & 1))) {
                            atomicExch(g.err, 13);
                            *aborted = 1;
                            break;
                        }
                        tc::fence_after_sync();
                        const uint64_t da = desc0 + (uint64_t)slot * slot_step;
                        const uint64_t db = da + (uint64_t)(CRT_SA >> 4);
                        for (int j = 0; j < nsub; ++j)
                            tc::mma_i8<CRT_IDESC>(acc, da + (uint64_t)(j * (CRT_ATILE >> 4)),
                                                  db + (uint64_t)(j * (CRT_BTILE >> 4)), (kb + j) > 0 ? 1u : 0u);
                        tc::mma_commit(&empty[slot]);
                    }
                    if (*aborted) break;
                    tc::mma_commit(&accfull[buf]);
                }
            }
        }
    } else {
        // epilogue warps
        auto wait_full = [&](int buf, uint32_t parity) { return tc::mbar_wait(&accfull[buf], parity); };
        auto release = [&](int buf) { tc::mbar_arrive(&accempty[buf]); };
        long long u = 0;
        for (int tile = blockIdx.x; tile < g.ntiles; tile += gridDim.x) {
            const int cb = tile % g.CB, rb = (tile / g.CB) % g.RB, b = tile / (g.CB * g.RB);
            if (!crt_extract_tile(g, tmem, rb, cb, b, u, aborted, wait_full, release)) {
                *aborted = 1;
                break;
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 512u);
}

// ---------------------------------------------------------------- CTA-pair MMA kernel
// The same product with 256 x 256 output tiles on a cluster of two CTAs
// (tcgen05 cta_group::2): the even CTA's MMA thread issues 256 x 256 x 32
// MMAs whose A rows 0-127 and B columns 0-127 come from its own shared memory
// and A rows 128-255 and B columns 128-255 from the odd CTA's, at the same
// offsets; each CTA's TMEM receives its 128 rows.  Per SM and K step a CTA
// stages 4 KB of A and 4 KB of B for 128 x 256 multiply-adds where the
// single-CTA tile stages 4 + 8 KB, so the copies per multiply-add drop by a
// third.  Measured it is the slower of the two (1874 against 2187 int8 TOPS
// at 1250^3 x 8 with four K steps per stage; neither the copies nor shared-
// memory bandwidth bound the single-CTA kernel, whose MMA stream probes at
// full rate beside concurrent copies), so it is opt-in (sc_crt_tiles_set).
// Both CTAs load their halves with 2-D tensor copies (cta_group::2, each
// into its own CTA only) that complete on the even CTA's stage barrier, which expects the
// bytes of both; the MMA thread's commits arrive on the barriers of both CTAs
// (one commit per CTA).  Each CTA's epilogue warps drain its own TMEM rows as
// in the single-CTA kernel and release the accumulator on the even CTA's
// barrier.  Every wait is bounded and gives up once either CTA has aborted; a
// CTA that aborts raises the other's flag through distributed shared memory.
constexpr int C2_BTILE = CRT_BTILE / 2;             // 128 columns x 32 K bytes
constexpr int C2_SA = CRT_KSUB * CRT_ATILE;         // 24 KB
constexpr int C2_SB = CRT_KSUB * C2_BTILE;          // 24 KB
constexpr int C2_SLOT = C2_SA + C2_SB;              // 48 KB
constexpr int C2_NS = (192 * 1024) / C2_SLOT;      // ring slots (192 KB)
constexpr int C2_ROW = 256;                         // bytes per row of the tensor maps (box 256 x 96 = one stage)
static_assert(C2_SA % C2_ROW == 0 && C2_SA / C2_ROW <= 256, "tensor box rows");
static_assert(CRT_NS * CRT_SLOT + 1024 <= 227 * 1024 && C2_NS * C2_SLOT + 1024 <= 227 * 1024, "shared memory");
constexpr uint32_t C2_IDESC = tc::idesc_i8(2 * CRT_BM, CRT_BN);

__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(CRT_THREADS, 1)
    crt_mma2_kernel(CrtArgs g, const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t full[C2_NS], empty[C2_NS], accfull[2], accempty[2], done;
    __shared__ uint32_t tmem_base;
    __shared__ int abort_flag;
    volatile int* aborted = &abort_flag;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t rank = tc::cluster_rank();
    const bool leader = rank == 0;
    const int pair = (int)(blockIdx.x >> 1), npairs = (int)(gridDim.x >> 1);
    const int KB = g.KB, RB2 = g.RB >> 1;

    if (threadIdx.x == 0) {
        for (int q = 0; q < C2_NS; ++q) {
            tc::mbar_init(&full[q], 1);
            tc::mbar_init(&empty[q], 1);
        }
        for (int q = 0; q < 2; ++q) {
            tc::mbar_init(&accfull[q], 1);
            tc::mbar_init(&accempty[q], 2 * CRT_EPI_WARPS);
        }
        tc::mbar_init(&done, 1);
        *aborted = 0;
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) tc::tmem_alloc2(&tmem_base, 512u);
    tc::fence_before_sync();
    tc::cluster_sync();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_base;
    const uint32_t peer_abort = tc::peer_addr(&abort_flag, rank ^ 1u);
    auto abort_pair = [&](int code) {
        if (!*aborted) atomicExch(g.err, code);
        *aborted = 1;
        tc::st_remote_u32(peer_abort, 1u);
    };
    // bounded wait that also gives up when either CTA has aborted
    auto wait = [&](uint64_t* bar, uint32_t parity) -> bool {
        if (tc::mbar_try_cluster(bar, parity)) return true;
        const unsigned long long t0 = tc::globaltimer_ns();
        for (long long it = 0; it < tc::TC_SPIN; ++it) {
            if (tc::mbar_try_cluster(bar, parity)) return true;
            if (*aborted || tc::globaltimer_ns() - t0 > tc::TC_TIMEOUT_NS) return false;
        }
        return false;
    };
    const long long planeA = (long long)g.RB * KB * CRT_ATILE;
    const long long planeB = (long long)g.CB * KB * CRT_BTILE;

    if (warp == 0) {
        if (lane == 0) {
            // producer (both CTAs): this CTA's 128 rows of A and 128 columns of B, one box each per stage
            // (a stage of fewer than CRT_KSUB K steps loads the whole box; the MMAs skip the rest)
            long long stage = 0;
            for (int tile = pair; tile < g.ntiles && !*aborted; tile += npairs) {
                const int cb = tile % g.CB, rb2 = (tile / g.CB) % RB2, b = tile / (g.CB * RB2);
                const int rb = 2 * rb2 + (int)rank, cbh = 2 * cb + (int)rank;
                for (int t = 0; t < CRT_NMOD && !*aborted; ++t) {
                    const long long offA = ((long long)b * CRT_NMOD + t) * planeA + (long long)rb * KB * CRT_ATILE;
                    const long long offB = ((long long)b * CRT_NMOD + t) * planeB + (long long)cbh * KB * C2_BTILE;
                    for (int kb = 0; kb < KB; kb += CRT_KSUB, ++stage) {
                        const int slot = (int)(stage % C2_NS);
                        if (stage >= C2_NS && !wait(&empty[slot], (uint32_t)(((stage / C2_NS) - 1) & 1))) {
                            abort_pair(21);
                            break;
                        }
                        const uint32_t bar = tc::peer_addr(&full[slot], 0u);
                        if (leader) tc::mbar_expect_tx(&full[slot], (uint32_t)(2 * C2_SLOT));
                        unsigned char* sa = smem_raw + (size_t)slot * C2_SLOT;
                        tc::tma2d_pair(sa, &tmA, 0, (int)((offA + (long long)kb * CRT_ATILE) / C2_ROW), bar);
                        tc::tma2d_pair(sa + C2_SA, &tmB, 0, (int)((offB + (long long)kb * C2_BTILE) / C2_ROW), bar);
                    }
                }
            }
            // drain: the copies of both CTAs complete on the even CTA's barriers
            if (leader)
                for (long long s2 = (stage > C2_NS ? stage - C2_NS : 0); s2 < stage; ++s2)
                    tc::mbar_wait(&full[s2 % C2_NS], (uint32_t)((s2 / C2_NS) & 1));
        }
    } else if (warp == 1) {
        if (lane == 0 && leader) {
            // MMA issuer of the pair
            const uint64_t desc0 = tc::smem_desc(smem_raw);
            const uint64_t slot_step = (uint64_t)(C2_SLOT >> 4);
            long long stage = 0, u = 0;
            for (int tile = pair; tile < g.ntiles && !*aborted; tile += npairs) {
                for (int t = 0; t < CRT_NMOD && !*aborted; ++t, ++u) {
                    const int buf = (int)(u & 1);
                    if (u >= 2 && !wait(&accempty[buf], (uint32_t)(((u >> 1) - 1) & 1))) {
                        abort_pair(22);
                        break;
                    }
                    tc::fence_after_sync();
                    const uint32_t acc = tmem + (uint32_t)(buf * CRT_BN);
                    for (int kb = 0; kb < KB; kb += CRT_KSUB, ++stage) {
                        const int nsub = min(CRT_KSUB, KB - kb);
                        const int slot = (int)(stage % C2_NS);
                        if (!wait(&full[slot], (uint32_t)((stage / C2_NS) & 1))) {
                            abort_pair(23);
                            break;
                        }
                        tc::fence_after_sync();
                        const uint64_t da = desc0 + (uint64_t)slot * slot_step;
                        const uint64_t db = da + (uint64_t)(C2_SA >> 4);
                        for (int j = 0; j < nsub; ++j)
                            tc::mma2_i8<C2_IDESC>(acc, da + (uint64_t)(j * (CRT_ATILE >> 4)),
                                                  db + (uint64_t)(j * (C2_BTILE >> 4)), (kb + j) > 0 ? 1u : 0u);
                        tc::mma2_commit(tc::smem_u32(&empty[slot]));
                        tc::mma2_commit(tc::peer_addr(&empty[slot], 1u));
                    }
                    if (*aborted) break;
                    tc::mma2_commit(tc::smem_u32(&accfull[buf]));
                    tc::mma2_commit(tc::peer_addr(&accfull[buf], 1u));
                }
            }
            // every MMA issued must have completed before either CTA releases its TMEM or shared memory
            tc::mma2_commit(tc::smem_u32(&done));
            if (!tc::mbar_wait(&done, 0)) atomicExch(g.err, 25);
        }
    } else {
        // epilogue warps: this CTA's 128 rows of each 256-row tile
        auto wait_full = [&](int buf, uint32_t parity) { return wait(&accfull[buf], parity); };
        auto release = [&](int buf) { tc::mbar_arrive_remote(tc::peer_addr(&accempty[buf], 0u)); };
        long long u = 0;
        for (int tile = pair; tile < g.ntiles; tile += npairs) {
            const int cb = tile % g.CB, rb2 = (tile / g.CB) % RB2, b = tile / (g.CB * RB2);
            if (!crt_extract_tile(g, tmem, 2 * rb2 + (int)rank, cb, b, u, aborted, wait_full, release)) {
                if (lane == 0) abort_pair(14);
                break;
            }
        }
    }
    __syncwarp();
    tc::fence_before_sync();
    tc::cluster_sync();
    tc::fence_after_sync();
    if (warp == 0) tc::tmem_dealloc2(tmem, 512u);
}

// 2-D byte tensor over a packed operand buffer: rows of 256 bytes, boxes of
// 256 x C2_SA / 256 rows (one stage); the driver's encoder comes through the runtime
// (no link against the driver library)
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        (void)cudaGetLastError();
        return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
    }();
    return fn;
}
bool byte_tensor_map(CUtensorMap* map, const void* base, size_t bytes) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = tensor_map_encoder();
    if (!enc || bytes % C2_ROW != 0 || (reinterpret_cast<uintptr_t>(base) & 15) != 0) return false;
    const cuuint64_t dims[2] = {(cuuint64_t)C2_ROW, (cuuint64_t)(bytes / C2_ROW)};
    const cuuint64_t strides[1] = {(cuuint64_t)C2_ROW};
    const cuuint32_t box[2] = {(cuuint32_t)C2_ROW, (cuuint32_t)(C2_SA / C2_ROW)};
    const cuuint32_t estr[2] = {1, 1};
    return enc(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void*>(base), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// per device: constants copied, kernel limits raised, CTA-pair capacity found
std::mutex g_crt_mu;
bool g_crt_const_ready[64] = {};
int g_crt_pairs[64] = {};

// int8 tensor-core throughput probe: one CTA per SM issues `iters` MMAs of
// 128 x 256 x 32 (the modular engine's shape) on operands resident in shared
// memory into one TMEM accumulator, then waits (bounded) for them
__global__ void __launch_bounds__(128, 1) int8_probe_kernel(int iters, int* err) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ __align__(8) uint64_t done;
    __shared__ uint32_t tmem_base;
    const int warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < CRT_STAGE / 16; i += blockDim.x)
        reinterpret_cast<uint4*>(smem_raw)[i] = make_uint4(0x01010101u, 0u, 0x01010101u, 0u);
    if (threadIdx.x == 0) {
        tc::mbar_init(&done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) tc::tmem_alloc(&tmem_base, 256u);
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_base;
    if (threadIdx.x == 32) {
        const uint64_t da = tc::smem_desc(smem_raw);
        const uint64_t db = da + (uint64_t)(CRT_ATILE >> 4);
        for (int it = 0; it < iters; ++it) tc::mma_i8<CRT_IDESC>(tmem, da, db, it > 0 ? 1u : 0u);
        tc::mma_commit(&done);
    }
    bool ok = tc::mbar_wait(&done, 0);
    if (!ok && threadIdx.x == 0) atomicExch(err, 1);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 256u);
}

}  // namespace

sc_status int8_peak_probe(int device, Workspace& ws, double* tops) {
    int sms = 148;
    SC_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    int* err;
    SC_TRY(ws.get(&err, 1, WS_OZ_ERR, 0));
    SC_CUDA_TRY(cudaMemset(err, 0, sizeof(int)));
    SC_CUDA_TRY(cudaFuncSetAttribute(int8_probe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, CRT_STAGE + 1024));
    const int iters = 8192;
    cudaEvent_t e0, e1;
    SC_CUDA_TRY(cudaEventCreate(&e0));
    SC_CUDA_TRY(cudaEventCreate(&e1));
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(e0, 0);
        int8_probe_kernel<<<sms, 128, CRT_STAGE + 1024>>>(iters, err);
        count_launch();
        cudaEventRecord(e1, 0);
        SC_CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int herr = 0;
    SC_CUDA_TRY(cudaMemcpy(&herr, err, sizeof(int), cudaMemcpyDeviceToHost));
    if (herr) {
        set_error("int8 probe: tensor-core wait timed out");
        return SC_CUDA_ERROR;
    }
    const double ops = 2.0 * CRT_BM * CRT_BN * CRT_BK * (double)iters * sms;
    *tops = ops / (best * 1e-3) / 1e12;
    return SC_OK;
}

// packed bytes of the residue operands per batch entry (row tiles rounded up
// to an even count, as the CTA-pair kernel needs)
size_t crt_packed_bytes(int m, int n, int k) {
    const long long RB = 2 * ((2LL * m + 2 * CRT_BM - 1) / (2 * CRT_BM)), CB = ((long long)n + CRT_BN - 1) / CRT_BN,
                    KB = (2LL * k + CRT_BK - 1) / CRT_BK;
    return (size_t)CRT_NMOD * (size_t)KB * ((size_t)RB * CRT_ATILE + (size_t)CB * CRT_BTILE);
}

sc_status zgemm_crt(cudaStream_t st, const GemmArgs& g, int batch, Workspace& ws, int* err) {
    if (g.m <= 0 || g.n <= 0 || batch <= 0) return SC_OK;
    if (!err) {
        set_error("zgemm_crt: no error word");
        return SC_BADINPUT;
    }
    if (2LL * g.k * 128 * 128 >= (1LL << 31)) {
        set_error("zgemm_crt: K = %d too deep for exact int32 accumulation", g.k);
        return SC_BADINPUT;
    }
    int dev = 0;
    SC_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) {
        set_error("zgemm_crt: device %d out of range", dev);
        return SC_BADINPUT;
    }
    static const CrtConst host_const = make_constants();
    std::unique_lock<std::mutex> init_lock(g_crt_mu);
    if (!g_crt_const_ready[dev]) {
        SC_CUDA_TRY(cudaMemcpyToSymbol(c_crt, &host_const, sizeof(CrtConst)));
        SC_TRY(smem_opt_in(crt_mma_kernel, CRT_NS * CRT_SLOT + 1024));
        const bool pair_ok = cudaFuncSetAttribute(crt_mma2_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  C2_NS * C2_SLOT + 1024) == cudaSuccess;
        if (!pair_ok) (void)cudaGetLastError();
        // clusters of two that fit on the device at once (SMs left without a
        // partner in their GPC cannot hold one): the pair kernel's grid
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(2, 1, 1);
        cfg.blockDim = dim3(CRT_THREADS, 1, 1);
        cfg.dynamicSmemBytes = C2_NS * C2_SLOT + 1024;
        int ncl = 0;
        if (!pair_ok || cudaOccupancyMaxActiveClusters(&ncl, crt_mma2_kernel, &cfg) != cudaSuccess) {
            ncl = 0;                 // no CTA pairs: the single-CTA tiles serve every product
            (void)cudaGetLastError();
        }
        g_crt_pairs[dev] = ncl;
        g_crt_const_ready[dev] = true;
    }
    const int npairs = g_crt_pairs[dev];
    init_lock.unlock();
    int sms = 148;
    SC_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const int bits = crt_bits(g.k, host_const.log2P);
    const bool pair = ws.crt_tiles != 0 && npairs > 0;
    const int RB = pair ? 2 * ((2 * g.m + 2 * CRT_BM - 1) / (2 * CRT_BM)) : (2 * g.m + CRT_BM - 1) / CRT_BM,
              CB = (g.n + CRT_BN - 1) / CRT_BN, KB = (2 * g.k + CRT_BK - 1) / CRT_BK;
    if (RB > 65535 || KB > 65535) {
        set_error("zgemm_crt: grid too large");
        return SC_BADINPUT;
    }
    // sub-batches so that the packed operands and the residues stay within 8 GiB
    const size_t res_per = (size_t)CRT_NMOD * RB * CRT_BM * (size_t)CB * CRT_BN;
    const size_t per = crt_packed_bytes(g.m, g.n, g.k) + res_per;
    int sub = (int)std::max<size_t>(1, std::min<size_t>((size_t)batch, (8ULL << 30) / std::max<size_t>(per, 1)));
    if (sub > 65535) sub = 65535;
    int8_t *Aq, *Bq, *res;
    int* ex;
    const size_t aq = (size_t)sub * CRT_NMOD * RB * KB * CRT_ATILE;
    const size_t bq = (size_t)sub * CRT_NMOD * CB * KB * CRT_BTILE;
    SC_TRY(ws.get(&Aq, aq, WS_OZ_A, st));
    SC_TRY(ws.get(&Bq, bq, WS_OZ_B, st));
    SC_TRY(ws.get(&ex, (size_t)batch * (g.m + g.n), WS_OZ_E, st));
    SC_TRY(ws.get(&res, (size_t)sub * res_per, WS_CRT_RES, st));
    int* rowexp = ex;
    int* colexp = ex + (size_t)batch * g.m;
    size_t mark_all = 0;
    if (ws.time_kernels)
        SC_TRY(ws.mark_begin(st, 3, 8.0 * g.m * (double)g.n * g.k * batch, 0.0, &mark_all));
    SC_CUDA_TRY(cudaMemsetAsync(rowexp, 0x80, sizeof(int) * (size_t)batch * g.m, st));
    SC_TRY(oz_exponents(st, g, batch, rowexp, colexp));
    for (int b0 = 0; b0 < batch; b0 += sub) {
        const int nb = std::min(sub, batch - b0);
        GemmArgs h = g;
        if (g.Ap) h.Ap = g.Ap + b0; else h.A = g.A + (long long)b0 * g.sA;
        if (g.Bp) h.Bp = g.Bp + b0; else h.B = g.B + (long long)b0 * g.sB;
        crt_pack_a_kernel<<<dim3(RB, KB, nb), 256, 0, st>>>(g.m, g.k, h.A, h.Ap, g.lda, g.sA,
                                                           rowexp + (size_t)b0 * g.m, bits, RB, KB, Aq);
        crt_pack_b_kernel<<<dim3(4 * CB, KB, nb), 256, 0, st>>>(g.k, g.n, h.B, h.Bp, g.ldb, g.sB,
                                                           colexp + (size_t)b0 * g.n, bits, CB, KB, pair ? 1 : 0,
                                                           Bq);
        count_launch(2);
        SC_CHECK_LAUNCH("crt pack");
        CrtArgs a;
        a.m = g.m;
        a.n = g.n;
        a.k = g.k;
        a.RB = RB;
        a.CB = CB;
        a.KB = KB;
        a.batch = nb;
        a.ntiles = nb * (pair ? RB / 2 : RB) * CB;
        a.shift = 2 * bits;
        a.Aq = Aq;
        a.Bq = Bq;
        a.rowexp = rowexp + (size_t)b0 * g.m;
        a.colexp = colexp + (size_t)b0 * g.n;
        a.alpha = g.alpha;
        a.beta = g.beta;
        a.alphas = g.alphas ? g.alphas + b0 : nullptr;
        a.C = g.Cp ? nullptr : g.C + (long long)b0 * g.sC;
        a.Cp = g.Cp ? g.Cp + b0 : nullptr;
        a.ldc = g.ldc;
        a.sC = g.sC;
        a.res = res;
        a.Mp = RB * CRT_BM;
        a.Np = CB * CRT_BN;
        a.err = err;
        size_t mark = 0;
        if (ws.time_kernels) {
            const double macs = (double)CRT_NMOD * nb * (double)RB * CRT_BM * (double)CB * CRT_BN * (double)KB * CRT_BK;
            SC_TRY(ws.mark_begin(st, 2, 8.0 * g.m * (double)g.n * g.k * nb, 2.0 * macs, &mark));
        }
        CUtensorMap tmA, tmB;
        if (pair && (!byte_tensor_map(&tmA, Aq, (size_t)nb * CRT_NMOD * RB * KB * CRT_ATILE) ||
                     !byte_tensor_map(&tmB, Bq, (size_t)nb * CRT_NMOD * CB * KB * CRT_BTILE))) {
            set_error("zgemm_crt: tensor map of the packed operands could not be encoded");
            return SC_CUDA_ERROR;
        }
        if (pair) {
            // two CTAs per tile, at most one CTA per SM
            const int grid = 2 * std::min(a.ntiles, std::min(npairs, sms / 2));
            crt_mma2_kernel<<<grid, CRT_THREADS, C2_NS * C2_SLOT + 1024, st>>>(a, tmA, tmB);
        } else {
            const int grid = std::min(a.ntiles, sms);
            crt_mma_kernel<<<grid, CRT_THREADS, CRT_NS * CRT_SLOT + 1024, st>>>(a);
        }
        count_launch();
        if (ws.time_kernels) SC_TRY(ws.mark_end(st, mark));
        SC_CHECK_LAUNCH("crt mma");
        crt_rebuild_kernel<<<dim3((g.n + 255) / 256, (g.m + 7) / 8, nb), 256, 0, st>>>(a);
        count_launch();
        SC_CHECK_LAUNCH("crt rebuild");
    }
    if (ws.time_kernels) SC_TRY(ws.mark_end(st, mark_all));
    return SC_OK;
}

}  // namespace sc
