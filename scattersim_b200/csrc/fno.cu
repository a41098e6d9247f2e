// Fourier-neural-operator surrogate of the thin-volume solve: a 64 x 64 index
// map plus the wavelength in, the R/T amplitudes of the 11 x 11 orders out
// (the x vector of ScatterVolume.cpp:739 for --coef 11 11).  The plain solve is
// its training data, its fallback and the measure of its error.
//
// Network (width W = 64, 4 spectral layers, 16 x 16 retained modes):
//   in  = [n(x, y), (lambda - 0.6) / 0.2, x / 63, y / 63,
//          cos phi, sin phi], phi = 2 pi n d / lambda                   6 x 64 x 64
//         (phi is the thin-element phase through the d = 1 um slab: its
//         mean over the cell is the zero-order transmission to first order)
//   v0  = P in + bP                                                   lift
//   u_l = W_l v_l + b_l + Re IDFT(M_l . DFT(v_l)),  v_{l+1} = GELU(u_l)
//         (no GELU after the last layer); DFT keeps kx in [-16, 16),
//         ky in [0, 16) (512 complex modes), M_l is a complex W x W
//         matrix per mode, IDFT is the real inverse of that half spectrum
//   h   = GELU(Q1 v4 + bQ1) (128 channels), o = Q2 h + bQ2 (12 channels)
//   amplitudes of channel pair c: sum_xy (o_2c + i o_2c+1) e^-i theta / 4096
//         at the 121 orders, theta = 2 pi (p x + q y) / 64, p, q in [-5, 5]
// Every linear map (lift, pointwise, the truncated DFT and its real inverse
// as separable partial DFTs -- along y, then x; back along x, then y -- the
// per-mode mixing, projections, readout) is one hand-written tensor-core GEMM: operands rounded to BF16 as they are staged,
// tcgen05.mma kind::f16 with FP32 accumulation in tensor memory, FP32 in global
// memory, arbitrary strides and batches.  Training: relative squared error per sample, Adam on
// FP32 master weights.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include <cuda_bf16.h>

#include "common.cuh"
#include "kernels.cuh"
#include "tcgen05.cuh"

namespace sc {
namespace fno {

constexpr int G = 64;                 // grid side
constexpr int NP = G * G;             // pixels
constexpr int W = 64;                 // width
constexpr int CIN = 6;                // input channels
constexpr float SLAB_UM = 1.0f;       // slab thickness of the workload (um)
constexpr int L = 4;                  // spectral layers
constexpr int MX = 16, MY = 16;       // retained modes: kx in [-MX, MX), ky in [0, MY)
constexpr int NM = 2 * MX * MY;       // 512 complex modes
constexpr int NF = 2 * NM;            // 1024 real columns: [re | im]
constexpr int SEP = G * 2 * MY;       // 2048: one channel after the y transform (64 x [re 16 | im 16])
constexpr int HID = 128;              // projection hidden channels
constexpr int COUT = 12;              // 6 complex output fields
constexpr int NO = 11;                // orders per axis
constexpr int NORD = NO * NO;         // 121
constexpr int NOUT = 6 * NORD * 2;    // 1452 reals per sample
constexpr int PW = 2 * NORD + 2;      // 244: readout columns [cos | sin] padded with zeros to a multiple of 4,
                                      // so that the readout products take the vector operand loads
// separable-transform operators, packed in one buffer
constexpr int OP_FY = 0, OP_EX = OP_FY + G * 2 * MY, OP_ER = OP_EX + G * G, OP_EI = OP_ER + G * G,
              OP_GY = OP_EI + G * G, OP_TOTAL = OP_GY + 2 * MY * G;

// ------------------------------------------------------------------ BF16 GEMM
// C_b[m, n] = alpha * sum_k A_b[m, k] B_b[k, n] + beta * C_b[m, n], element
// addresses A + b sAb + m sAm + k sAk (likewise B, C).
struct Gemm {
    int m, n, k, batch;
    float alpha, beta;
    const float* A;
    long long sAm, sAk, sAb;
    const float* B;
    long long sBk, sBn, sBb;
    float* C;
    long long sCm, sCn, sCb;
    // split-K: batch entry b, K chunk s (of kchunk values) writes output entry
    // b * ksplit + s; ksplit = 1 is the plain batched product
    int ksplit = 1, kchunk = 0;
};

// Tile of the tensor-core GEMM: 128 rows (the TMEM lanes) x 64 columns,
// staged 32 K values at a time.  Operands are FP32 in global memory, rounded
// to BF16 as the CTA writes them into shared memory in the UMMA K-major
// core-matrix layout (8 rows x 16 bytes per core matrix, LBO = 128 B along K,
// SBO = 512 B between 8-row groups); one thread issues two tcgen05.mma
// kind::f16 (BF16 x BF16 -> FP32, 128 x 64 x 16) per stage into a TMEM
// accumulator; two shared-memory stages let the CTA convert and store the
// next K slice while the tensor core consumes the current one (an mbarrier
// per stage, signalled by tcgen05.commit).  The epilogue reads the
// accumulator with tcgen05.ld and writes C with its strides.  Every wait is
// bounded; a timeout sets the context's error word.
constexpr int TM = 128, TN = 64, TK = 32, GT = 128;
constexpr int UA_BYTES = TM * TK * 2, UB_BYTES = TN * TK * 2;   // 8 KB, 4 KB per stage
constexpr uint32_t U_IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) |
                             ((uint32_t)(TM >> 4) << 24);      // F32 accumulate, A = B = BF16, K-major

// byte offset of (row, k) in a K-major BF16 core-matrix tile of TK = 32 columns
__device__ __forceinline__ int uoff(int r, int kk) { return (r >> 3) * 512 + (kk >> 3) * 128 + (r & 7) * 16 + (kk & 7) * 2; }

__device__ __forceinline__ uint64_t udesc(const void* p) {
    return (uint64_t)((tc::smem_u32(p) >> 4) & 0x3FFF) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(512 >> 4) << 32) |
           (1ULL << 46);
}
__device__ __forceinline__ void umma_bf16(uint32_t dtmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(dtmem), "l"(adesc),
        "l"(bdesc), "r"(U_IDESC), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}
__device__ __forceinline__ uint32_t bf2(float a, float b) {
    const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t*>(&v);
}

// operand load modes: 1 float4 along k (stride_k == 1; the host picks it only
// when the base is 16-byte aligned, the row and batch strides are multiples of
// 4 and k is), otherwise scalar loads (0: any strides, 2: the row index
// contiguous, where the scalar loads of a warp coalesce).  A thread stages
// 16-byte units, one row x 8 K values each; consecutive threads take
// consecutive rows, so a warp's loads in mode 2 read contiguous rows and its
// 16-byte shared-memory stores (8 consecutive rows of a core matrix, 128 B)
// are free of bank conflicts.
template <int V, int R>
struct Stager {
    static constexpr int U = R * (TK / 8) / GT;   // units per thread
    float v[U][8];
    __device__ __forceinline__ void load(const float* X, long long s_r, long long s_k, int rows, int kdim, int r0,
                                         int k0, int tid) {
#pragma unroll
        for (int i = 0; i < U; ++i) {
            const int u = tid + GT * i;
            const int r = u % R, o = u / R;
            const int gr = r0 + r, gk = k0 + 8 * o;
            if constexpr (V == 1) {
                float4 x0 = make_float4(0.f, 0.f, 0.f, 0.f), x1 = x0;
                if (gr < rows) {
                    const float* p = X + gr * s_r + gk;
                    if (gk < kdim) x0 = *reinterpret_cast<const float4*>(p);
                    if (gk + 4 < kdim) x1 = *reinterpret_cast<const float4*>(p + 4);
                }
                v[i][0] = x0.x;
                v[i][1] = x0.y;
                v[i][2] = x0.z;
                v[i][3] = x0.w;
                v[i][4] = x1.x;
                v[i][5] = x1.y;
                v[i][6] = x1.z;
                v[i][7] = x1.w;
            } else {
#pragma unroll
                for (int j = 0; j < 8; ++j)
                    v[i][j] = (gr < rows && gk + j < kdim) ? X[gr * s_r + (long long)(gk + j) * s_k] : 0.f;
            }
        }
    }
    __device__ __forceinline__ void store(unsigned char* tile, int tid) const {
#pragma unroll
        for (int i = 0; i < U; ++i) {
            const int u = tid + GT * i;
            const int r = u % R, o = u / R;
            *reinterpret_cast<uint4*>(tile + uoff(r, 8 * o)) =
                make_uint4(bf2(v[i][0], v[i][1]), bf2(v[i][2], v[i][3]), bf2(v[i][4], v[i][5]), bf2(v[i][6], v[i][7]));
        }
    }
};

// set by a tensor-core GEMM whose pipeline wait timed out; read and cleared by sc_fno_status
__device__ int g_fno_err;

template <int VA, int VB>
__global__ void __launch_bounds__(GT) bf16_gemm_kernel(Gemm g) {
    __shared__ __align__(1024) unsigned char sm[2][UA_BYTES + UB_BYTES];
    __shared__ __align__(8) uint64_t mma_bar[2], done_bar;
    __shared__ uint32_t tmem_base;
    const int z = blockIdx.z;
    const int b = z / g.ksplit, kbeg = (z - b * g.ksplit) * g.kchunk;
    const int kdim = min(g.k - kbeg, g.kchunk);
    const float* A = g.A + b * g.sAb + (long long)kbeg * g.sAk;
    const float* B = g.B + b * g.sBb + (long long)kbeg * g.sBk;
    float* C = g.C + z * g.sCb;
    const int m0 = blockIdx.x * TM, n0 = blockIdx.y * TN;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) {
        tc::mbar_init(&mma_bar[0], 1);
        tc::mbar_init(&mma_bar[1], 1);
        tc::mbar_init(&done_bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    if (warp == 0) tc::tmem_alloc(&tmem_base, 64u);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tmem_base;
    Stager<VA, TM> sa;
    Stager<VB, TN> sb;
    const int nk = kdim > 0 ? (kdim + TK - 1) / TK : 0;
    bool ok = true;
    if (nk > 0) {
        sa.load(A, g.sAm, g.sAk, g.m, kdim, m0, 0, tid);
        sb.load(B, g.sBn, g.sBk, g.n, kdim, n0, 0, tid);
    }
    for (int t = 0; t < nk; ++t) {
        const int s = t & 1;
        // the MMAs of K slice t - 2 read this stage: wait for them
        if (t >= 2 && !tc::mbar_wait(&mma_bar[s], (uint32_t)(((t - 2) >> 1) & 1))) ok = false;
        ok = __syncthreads_and(ok);
        if (!ok) break;
        sa.store(sm[s], tid);
        sb.store(sm[s] + UA_BYTES, tid);
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            const uint64_t da = udesc(sm[s]), db = udesc(sm[s] + UA_BYTES);
            umma_bf16(tmem, da, db, t > 0 ? 1u : 0u);
            umma_bf16(tmem, da + (256 >> 4), db + (256 >> 4), 1u);   // K 16..31: two core matrices on
            tc::mma_commit(&mma_bar[s]);
        }
        if (t + 1 < nk) {
            sa.load(A, g.sAm, g.sAk, g.m, kdim, m0, (t + 1) * TK, tid);
            sb.load(B, g.sBn, g.sBk, g.n, kdim, n0, (t + 1) * TK, tid);
        }
    }
    if (tid == 0) tc::mma_commit(&done_bar);
    bool ready = ok && tc::mbar_wait(&done_bar, 0);
    ready = __all_sync(0xffffffffu, ready);
    if (!ready && lane == 0) atomicExch(&g_fno_err, 1);
    tc::fence_after_sync();
    const int gm = m0 + warp * 32 + lane;
    if (g.sCn == 1 && g.sCm != 1) {
        // row-contiguous C: a thread's TMEM row goes through shared memory (the
        // operand stages are free: every MMA has completed) so that a warp
        // writes whole rows, 32 columns at a time; [128][33] floats, padded
        // against bank conflicts
        float* T = reinterpret_cast<float*>(&sm[0][0]);
        const bool vec = ((reinterpret_cast<uintptr_t>(C) & 15) == 0) && (g.sCm % 4 == 0);
        for (int c0 = 0; c0 < TN; c0 += 32) {
            uint32_t r[32];
            tc::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, r);
            __syncthreads();   // the previous half's rows have been written out
#pragma unroll
            for (int q = 0; q < 32; ++q) T[(warp * 32 + lane) * 33 + q] = nk > 0 ? g.alpha * __uint_as_float(r[q]) : 0.f;
            __syncthreads();
            if (ready) {
                // thread t: rows t / 8 + 16 i, columns 4 (t % 8) .. + 3
                const int cq = 4 * (tid & 7);
                const int gn = n0 + c0 + cq;
#pragma unroll 4
                for (int i = 0; i < 8; ++i) {
                    const int rr = (tid >> 3) + 16 * i;
                    const int row = m0 + rr;
                    if (row >= g.m) continue;
                    const float* t = T + rr * 33 + cq;
                    float* p = C + row * g.sCm + gn;
                    if (vec && gn + 3 < g.n) {
                        float4 v = make_float4(t[0], t[1], t[2], t[3]);
                        if (g.beta != 0.f) {
                            const float4 o = *reinterpret_cast<const float4*>(p);
                            v = make_float4(fmaf(g.beta, o.x, v.x), fmaf(g.beta, o.y, v.y), fmaf(g.beta, o.z, v.z),
                                            fmaf(g.beta, o.w, v.w));
                        }
                        *reinterpret_cast<float4*>(p) = v;
                    } else {
                        for (int q = 0; q < 4; ++q)
                            if (gn + q < g.n) p[q] = (g.beta == 0.f) ? t[q] : fmaf(g.beta, p[q], t[q]);
                    }
                }
            }
        }
    } else {
        for (int c0 = 0; c0 < TN; c0 += 32) {
            uint32_t r[32];
            tc::tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, r);
            if (ready && gm < g.m) {
#pragma unroll
                for (int q = 0; q < 32; ++q) {
                    const int gn = n0 + c0 + q;
                    if (gn < g.n) {
                        float* p = C + gm * g.sCm + gn * g.sCn;
                        const float v = nk > 0 ? g.alpha * __uint_as_float(r[q]) : 0.f;
                        *p = (g.beta == 0.f) ? v : fmaf(g.beta, *p, v);
                    }
                }
            }
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) tc::tmem_dealloc(tmem, 64u);
}

bool aligned16(const void* p) { return ((uintptr_t)p & 15) == 0; }

// vector mode of an operand with rows x cols = (mrows, k): 1 when k is
// contiguous, 2 when the row index is, 0 otherwise (see bf16_gemm_kernel)
int vec_mode(const float* base, long long s_row, long long s_k, long long s_batch, int rows, int k) {
    if (!aligned16(base) || s_batch % 4 != 0) return 0;
    if (s_k == 1 && s_row % 4 == 0 && k % 4 == 0) return 1;
    if (s_row == 1 && s_k % 4 == 0 && rows % 4 == 0) return 2;
    return 0;
}

template <int VA, int VB>
void launch_gemm(dim3 grid, cudaStream_t st, const Gemm& g) {
    bf16_gemm_kernel<VA, VB><<<grid, GT, 0, st>>>(g);
}

sc_status gemm(cudaStream_t st, const Gemm& g0) {
    if (g0.m <= 0 || g0.n <= 0 || g0.batch <= 0) return SC_OK;
    // the tile has 128 rows (TMEM lanes) and 64 columns: when n > m (the
    // network's products are mostly 64- or 12-row by thousands of columns)
    // compute C^T = B^T A^T so that the long dimension fills the rows
    // (and, for square shapes, when C is row-contiguous: the epilogue's
    // stores then run along the rows a warp covers)
    Gemm g = g0;
    if (g0.n > g0.m || (g0.n == g0.m && g0.sCn == 1 && g0.sCm != 1)) {
        g.m = g0.n;
        g.n = g0.m;
        g.A = g0.B;
        g.sAm = g0.sBn;
        g.sAk = g0.sBk;
        g.sAb = g0.sBb;
        g.B = g0.A;
        g.sBn = g0.sAm;
        g.sBk = g0.sAk;
        g.sBb = g0.sAb;
        g.sCm = g0.sCn;
        g.sCn = g0.sCm;
    }
    if (g.ksplit < 1 || (g.ksplit > 1 && g.k % (g.ksplit * TK) != 0)) {
        set_error("fno gemm: split-K needs k a multiple of 32 x ksplit");
        return SC_BADINPUT;
    }
    g.kchunk = g.k / g.ksplit;
    if ((long long)g.batch * g.ksplit > 65535 || (g.n + TN - 1) / TN > 65535) {
        set_error("fno gemm: grid too large");
        return SC_BADINPUT;
    }
    dim3 grid((g.m + TM - 1) / TM, (g.n + TN - 1) / TN, g.batch * g.ksplit);
    const int va = vec_mode(g.A, g.sAm, g.sAk, g.batch > 1 ? g.sAb : 0, g.m, g.k);
    const int vb = vec_mode(g.B, g.sBn, g.sBk, g.batch > 1 ? g.sBb : 0, g.n, g.k);
    switch (va * 3 + vb) {
        case 0: launch_gemm<0, 0>(grid, st, g); break;
        case 1: launch_gemm<0, 1>(grid, st, g); break;
        case 2: launch_gemm<0, 2>(grid, st, g); break;
        case 3: launch_gemm<1, 0>(grid, st, g); break;
        case 4: launch_gemm<1, 1>(grid, st, g); break;
        case 5: launch_gemm<1, 2>(grid, st, g); break;
        case 6: launch_gemm<2, 0>(grid, st, g); break;
        case 7: launch_gemm<2, 1>(grid, st, g); break;
        default: launch_gemm<2, 2>(grid, st, g); break;
    }
    count_launch();
    SC_CHECK_LAUNCH("fno gemm");
    return SC_OK;
}

// ------------------------------------------------------------------ elementwise
__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.f + erff(x * 0.70710678f)); }
__device__ __forceinline__ float gelu_grad(float x) {
    return 0.5f * (1.f + erff(x * 0.70710678f)) + x * 0.39894228f * expf(-0.5f * x * x);
}

// in[b] = [map, (lambda - 0.6) / 0.2, x / 63, y / 63, cos phi, sin phi]
__global__ void input_kernel(const float* __restrict__ maps, const float* __restrict__ lam, int Bn,
                             float* __restrict__ in) {
    const long long tot = (long long)Bn * NP;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
        const int b = (int)(t / NP), p = (int)(t % NP);
        float* o = in + (long long)b * CIN * NP;
        const float n = maps[t];
        o[p] = n;
        o[NP + p] = (lam[b] - 0.6f) / 0.2f;
        o[2 * NP + p] = (float)(p / G) / 63.f;
        o[3 * NP + p] = (float)(p % G) / 63.f;
        // phase in turns, reduced before the trigonometric call
        const float turns = n * SLAB_UM / lam[b];
        const float fr = turns - floorf(turns);
        float sv, cv;
        sincospif(2.f * fr, &sv, &cv);
        o[4 * NP + p] = cv;
        o[5 * NP + p] = sv;
    }
}

// x[b][c][p] += bias[c]; optionally a = GELU(x) (x keeps the pre-activation)
__global__ void bias_act_kernel(float* __restrict__ x, const float* __restrict__ bias, int C, int Bn, int act,
                                float* __restrict__ a) {
    const long long tot = (long long)Bn * C * NP;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
        const int c = (int)((t / NP) % C);
        const float v = x[t] + bias[c];
        x[t] = v;
        if (act) a[t] = gelu(v);
    }
}

// g *= GELU'(pre)
__global__ void gelu_back_kernel(float* __restrict__ g, const float* __restrict__ pre, long long tot) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x)
        g[t] *= gelu_grad(pre[t]);
}

// bias gradient in two deterministic passes: partial[c][s] = sum over the
// samples b = s, s + NSPL, ... and all pixels of g[b][c][p] (one CTA each),
// then db[c] += sum_s partial[c][s] in order
constexpr int NSPL = 32;
constexpr int KSPLIT = 8;              // K chunks of the per-sample weight gradients (K = NP)
__global__ void bias_grad_part_kernel(const float* __restrict__ g, int C, int Bn, float* __restrict__ part) {
    __shared__ float red[8];
    const int c = blockIdx.x, sp = blockIdx.y;
    float s = 0.f;
    for (int b = sp; b < Bn; b += NSPL)
        for (int p = threadIdx.x; p < NP; p += blockDim.x) s += g[((long long)b * C + c) * NP + p];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.f;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) t += red[i];
        part[c * NSPL + sp] = t;
    }
}

__global__ void bias_grad_sum_kernel(const float* __restrict__ part, int C, float* __restrict__ db) {
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= C) return;
    float t = 0.f;
    for (int sp = 0; sp < NSPL; ++sp) t += part[c * NSPL + sp];
    db[c] += t;
}

// out[i] += sum_r part[r][i] over R partials (per sample and K chunk): a block
// of 8 warps per 32 outputs, lanes along i (coalesced), warps splitting r,
// then a fixed-order sum across the warps (deterministic)
__global__ void __launch_bounds__(256) batch_sum_kernel(const float* __restrict__ part, int R, long long n,
                                                        float* __restrict__ out) {
    __shared__ float red[8][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long long i = blockIdx.x * 32LL + lane;
    float s = 0.f;
    if (i < n)
        for (int r = w; r < R; r += 8) s += part[(long long)r * n + i];
    red[w][lane] = s;
    __syncthreads();
    if (w == 0 && i < n) {
        float t = 0.f;
#pragma unroll
        for (int q = 0; q < 8; ++q) t += red[q][lane];
        out[i] += t;
    }
}
// out[b][i] = sum_s part[b S + s][i]: the K chunks of a split product, per sample
__global__ void ksum_kernel(const float* __restrict__ part, int S, int Bn, long long n, float* __restrict__ out) {
    const long long tot = (long long)Bn * n;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
        const long long b = t / n, i = t - b * n;
        float s = 0.f;
        for (int q = 0; q < S; ++q) s += part[(b * S + q) * n + i];
        out[t] = s;
    }
}
sc_status batch_sum(cudaStream_t st, const float* part, int R, long long n, float* out) {
    batch_sum_kernel<<<(unsigned)((n + 31) / 32), 256, 0, st>>>(part, R, n, out);
    count_launch();
    return SC_OK;
}

// readout: P[b][12][244] (cos | sin correlations, 2 zero columns) -> pred[b][6][121][re, im]
__global__ void readout_kernel(const float* __restrict__ P, int Bn, float* __restrict__ pred) {
    const int tot = Bn * 6 * NORD;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += gridDim.x * blockDim.x) {
        const int b = t / (6 * NORD), c = (t / NORD) % 6, j = t % NORD;
        const float* pr = P + ((long long)b * COUT + 2 * c) * PW;
        const float* pi = pr + PW;
        float* o = pred + (long long)b * NOUT + 2 * (c * NORD + j);
        o[0] = pr[j] + pi[NORD + j];
        o[1] = pi[j] - pr[NORD + j];
    }
}

// adjoint of readout_kernel
__global__ void readout_back_kernel(const float* __restrict__ dpred, int Bn, float* __restrict__ dP) {
    const int tot = Bn * 6 * NORD;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < tot; t += gridDim.x * blockDim.x) {
        const int b = t / (6 * NORD), c = (t / NORD) % 6, j = t % NORD;
        const float* d = dpred + (long long)b * NOUT + 2 * (c * NORD + j);
        float* pr = dP + ((long long)b * COUT + 2 * c) * PW;
        float* pi = pr + PW;
        pr[j] = d[0];
        pi[NORD + j] = d[0];
        pi[j] = d[1];
        pr[NORD + j] = -d[1];
    }
}

// x transform output U ([q][channel][32]: rows q = [cos kx; sin kx], columns
// [re ky | im ky] of the y transform) -> X (mode-major: X[md][channel] for the
// real parts md < 512, X[512 + md][channel] for the imaginary parts, mode md =
// r * 16 + ky):  Re = U[r][ky] + U[32+r][16+ky],  Im = U[r][16+ky] - U[32+r][ky]
__global__ void xcombine_kernel(const float* __restrict__ U, long long nch, float* __restrict__ X) {
    const long long tot = nch * NM;
    const long long qs = nch * 2 * MY;   // stride of q in U
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
        const long long c = t % nch;
        const int md = (int)(t / nch), r = md / MY, ky = md % MY;
        const float* u = U + c * 2 * MY;
        X[(long long)md * nch + c] = u[r * qs + ky] + u[(2 * MX + r) * qs + MY + ky];
        X[(long long)(NM + md) * nch + c] = u[r * qs + MY + ky] - u[(2 * MX + r) * qs + ky];
    }
}

// adjoint of xcombine_kernel
__global__ void xcombine_back_kernel(const float* __restrict__ dX, long long nch, float* __restrict__ dU) {
    const long long tot = nch * NM;
    const long long qs = nch * 2 * MY;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
        const long long c = t % nch;
        const int md = (int)(t / nch), r = md / MY, ky = md % MY;
        float* u = dU + c * 2 * MY;
        const float dr = dX[(long long)md * nch + c], di = dX[(long long)(NM + md) * nch + c];
        u[r * qs + ky] = dr;
        u[(2 * MX + r) * qs + MY + ky] = dr;
        u[r * qs + MY + ky] = di;
        u[(2 * MX + r) * qs + ky] = -di;
    }
}

// per-sample relative squared error; dpred = d loss / d pred; loss[b]
__global__ void loss_kernel(const float* __restrict__ pred, const float* __restrict__ tgt, int Bn,
                            float* __restrict__ dpred, float* __restrict__ loss) {
    __shared__ float r1[8], r2[8];
    const int b = blockIdx.x;
    const float* p = pred + (long long)b * NOUT;
    const float* y = tgt + (long long)b * NOUT;
    float e = 0.f, n = 0.f;
    for (int i = threadIdx.x; i < NOUT; i += blockDim.x) {
        const float d = p[i] - y[i];
        e += d * d;
        n += y[i] * y[i];
    }
    for (int o = 16; o > 0; o >>= 1) {
        e += __shfl_xor_sync(0xffffffffu, e, o);
        n += __shfl_xor_sync(0xffffffffu, n, o);
    }
    if ((threadIdx.x & 31) == 0) {
        r1[threadIdx.x >> 5] = e;
        r2[threadIdx.x >> 5] = n;
    }
    __syncthreads();
    float E = 0.f, N = 0.f;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) {
        E += r1[i];
        N += r2[i];
    }
    N = fmaxf(N, 1e-30f);
    if (threadIdx.x == 0) loss[b] = E / N;
    if (dpred)
        for (int i = threadIdx.x; i < NOUT; i += blockDim.x) dpred[(long long)b * NOUT + i] = 2.f * (p[i] - y[i]) / (N * Bn);
}

__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, long long n, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
        const float gi = g[t];
        const float mi = b1 * m[t] + (1.f - b1) * gi;
        const float vi = b2 * v[t] + (1.f - b2) * gi * gi;
        m[t] = mi;
        v[t] = vi;
        w[t] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

unsigned blocks(long long tot) {
    long long b = (tot + 255) / 256;
    if (b < 1) b = 1;
    if (b > 4096) b = 4096;
    return (unsigned)b;
}

sc_status bias_grad(cudaStream_t st, const float* g, int C, int Bn, float* db, float* part) {
    bias_grad_part_kernel<<<dim3(C, NSPL), 256, 0, st>>>(g, C, Bn, part);
    bias_grad_sum_kernel<<<(C + 127) / 128, 128, 0, st>>>(part, C, db);
    count_launch(2);
    return SC_OK;
}

// ------------------------------------------------------------------ parameters
struct Layout {
    long long P, bP, Wl[L], bl[L], SWr[L], SWi[L], Q1, bQ1, Q2, bQ2, total;
    Layout() {
        long long o = 0;
        auto take = [&](long long n) {
            long long r = o;
            o += (n + 63) / 64 * 64;
            return r;
        };
        P = take((long long)W * CIN);
        bP = take(W);
        for (int l = 0; l < L; ++l) {
            Wl[l] = take((long long)W * W);
            bl[l] = take(W);
            SWr[l] = take((long long)NM * W * W);
            SWi[l] = take((long long)NM * W * W);
        }
        Q1 = take((long long)HID * W);
        bQ1 = take(HID);
        Q2 = take((long long)COUT * HID);
        bQ2 = take(COUT);
        total = o;
    }
};

}  // namespace fno
}  // namespace sc

using namespace sc;
using namespace sc::fno;

struct sc_fno {
    int device = 0;
    int max_batch = 0;
    Layout lay;
    float *w = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;   // params, grads, Adam moments
    float *ops = nullptr, *R = nullptr;                               // DFT operators
    float *S1 = nullptr, *S2 = nullptr;                               // separable-transform scratch
    float *in = nullptr, *act[L + 1] = {}, *pre[L] = {}, *X[L] = {}, *Y = nullptr;
    float *hpre = nullptr, *h = nullptr, *o12 = nullptr, *P = nullptr, *pred = nullptr;
    float *dact = nullptr, *dv = nullptr, *dX = nullptr, *dY = nullptr, *dh = nullptr, *do12 = nullptr,
          *dP = nullptr, *dpred = nullptr, *part = nullptr, *loss = nullptr, *bpart = nullptr;
    long long step = 0;
};

namespace {

sc_status fno_alloc(float** p, long long n) {
    cudaError_t e = cudaMalloc(p, sizeof(float) * (size_t)(n > 0 ? n : 1));
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error("fno: device allocation of %lld floats failed", n);
        return SC_OOM;
    }
    return SC_OK;
}

// deterministic uniform [0, 1) stream (splitmix64)
struct Rng {
    uint64_t s;
    double next() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ULL);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    }
};

// wrapped signed frequency of retained row index r in [0, 2 MX)
int kx_of(int r) { return r < MX ? r : r - 2 * MX; }

// order index j (the solve's column-major (q, p) index) -> (p, q) in [-5, 5]
void order_pq(int j, int* p, int* q) {
    *q = j % NO - NO / 2;
    *p = j / NO - NO / 2;
}

Gemm mk(int m, int n, int k, int batch, float alpha, float beta, const float* A, long long sAm, long long sAk,
        long long sAb, const float* B, long long sBk, long long sBn, long long sBb, float* C, long long sCm,
        long long sCn, long long sCb) {
    return Gemm{m, n, k, batch, alpha, beta, A, sAm, sAk, sAb, B, sBk, sBn, sBb, C, sCm, sCn, sCb};
}
// the weight gradients contract over the 4096 pixels of one sample: split K
// into KSPLIT chunks (one partial per sample and chunk, summed by batch_sum),
// so that the product runs on Bn x KSPLIT CTAs instead of Bn
Gemm split_k(Gemm g) {
    g.ksplit = KSPLIT;
    return g;
}

// forward pass for Bn samples; keeps every activation for the backward pass
sc_status forward(sc_fno* f, const float* maps, const float* lam, int Bn, cudaStream_t st) {
    const Layout& Ly = f->lay;
    const float* w = f->w;
    const long long sv = (long long)W * NP;
    input_kernel<<<blocks((long long)Bn * NP), 256, 0, st>>>(maps, lam, Bn, f->in);
    count_launch();
    // lift: v0_b (W x NP) = P (W x CIN) in_b (CIN x NP)
    SC_TRY(gemm(st, mk(W, NP, CIN, Bn, 1.f, 0.f, w + Ly.P, CIN, 1, 0, f->in, NP, 1, (long long)CIN * NP, f->act[0], NP,
                       1, sv)));
    bias_act_kernel<<<blocks((long long)Bn * sv), 256, 0, st>>>(f->act[0], w + Ly.bP, W, Bn, 0, nullptr);
    count_launch();
    for (int l = 0; l < L; ++l) {
        float* vin = f->act[l];
        // truncated DFT: along y (batched over x: rows = channels, 64 y -> [re | im] 16),
        // then along x (one GEMM: [cos; sin] (64 x 64) times x by (channel, 32)),
        // combined into mode-major X
        const long long nch = (long long)Bn * W;
        SC_TRY(gemm(st, mk((int)nch, 2 * MY, G, G, 1.f, 0.f, vin, NP, 1, G, f->ops + OP_FY, 2 * MY, 1, 0, f->S1, 2 * MY,
                           1, nch * 2 * MY)));
        SC_TRY(gemm(st, mk(G, (int)(nch * 2 * MY), G, 1, 1.f, 0.f, f->ops + OP_EX, G, 1, 0, f->S1, nch * 2 * MY, 1, 0,
                           f->S2, nch * 2 * MY, 1, 0)));
        xcombine_kernel<<<blocks(nch * NM), 256, 0, st>>>(f->S2, nch, f->X[l]);
        count_launch();
        // per mode md: Y[md] (B x W) = X[md] (B x W) M[md] (W x W), complex as four real products
        const float* Xr = f->X[l];
        const float* Xi = f->X[l] + NM * nch;
        const float* Wr = w + Ly.SWr[l];
        const float* Wi = w + Ly.SWi[l];
        float* Yr = f->Y;
        float* Yi = f->Y + NM * nch;
        const long long ww = (long long)W * W;
        SC_TRY(gemm(st, mk(Bn, W, W, NM, 1.f, 0.f, Xr, W, 1, nch, Wr, W, 1, ww, Yr, W, 1, nch)));
        SC_TRY(gemm(st, mk(Bn, W, W, NM, -1.f, 1.f, Xi, W, 1, nch, Wi, W, 1, ww, Yr, W, 1, nch)));
        SC_TRY(gemm(st, mk(Bn, W, W, NM, 1.f, 0.f, Xr, W, 1, nch, Wi, W, 1, ww, Yi, W, 1, nch)));
        SC_TRY(gemm(st, mk(Bn, W, W, NM, 1.f, 1.f, Xi, W, 1, nch, Wr, W, 1, ww, Yi, W, 1, nch)));
        // u_b = W_l v_b + Y_b G + b_l
        float* u = f->pre[l];
        SC_TRY(gemm(st, mk(W, NP, W, Bn, 1.f, 0.f, w + Ly.Wl[l], W, 1, 0, vin, NP, 1, sv, u, NP, 1, sv)));
        // inverse: along x (Z[x][ky][channel] = [cos | -sin] Y and [sin | cos] Y,
        // one GEMM each over (ky, channel)), then along y into u (batched over x,
        // accumulated)
        SC_TRY(gemm(st, mk(G, (int)(MY * nch), G, 1, 1.f, 0.f, f->ops + OP_ER, G, 1, 0, f->Y, MY * nch, 1, 0, f->S1,
                           2 * MY * nch, 1, 0)));
        SC_TRY(gemm(st, mk(G, (int)(MY * nch), G, 1, 1.f, 0.f, f->ops + OP_EI, G, 1, 0, f->Y, MY * nch, 1, 0,
                           f->S1 + MY * nch, 2 * MY * nch, 1, 0)));
        SC_TRY(gemm(st, mk((int)nch, G, 2 * MY, G, 1.f, 1.f, f->S1, 1, nch, 2 * MY * nch, f->ops + OP_GY, G, 1, 0, u,
                           NP, 1, G)));
        const int act = (l < L - 1);
        bias_act_kernel<<<blocks((long long)Bn * sv), 256, 0, st>>>(u, w + Ly.bl[l], W, Bn, act, f->act[l + 1]);
        count_launch();
        if (!act)
            SC_CUDA_TRY(cudaMemcpyAsync(f->act[l + 1], u, sizeof(float) * Bn * sv, cudaMemcpyDeviceToDevice, st));
    }
    // projection
    const long long sh = (long long)HID * NP;
    SC_TRY(gemm(st, mk(HID, NP, W, Bn, 1.f, 0.f, w + Ly.Q1, W, 1, 0, f->act[L], NP, 1, sv, f->hpre, NP, 1, sh)));
    bias_act_kernel<<<blocks((long long)Bn * sh), 256, 0, st>>>(f->hpre, w + Ly.bQ1, HID, Bn, 1, f->h);
    count_launch();
    const long long so = (long long)COUT * NP;
    SC_TRY(gemm(st, mk(COUT, NP, HID, Bn, 1.f, 0.f, w + Ly.Q2, HID, 1, 0, f->h, NP, 1, sh, f->o12, NP, 1, so)));
    bias_act_kernel<<<blocks((long long)Bn * so), 256, 0, st>>>(f->o12, w + Ly.bQ2, COUT, Bn, 0, nullptr);
    count_launch();
    // readout correlations P_b (12 x 244) = o_b (12 x NP) R (NP x 244): K = NP split into KSPLIT chunks,
    // the partials summed per sample
    SC_TRY(gemm(st, split_k(mk(COUT, PW, NP, Bn, 1.f, 0.f, f->o12, NP, 1, so, f->R, PW, 1, 0, f->part, PW, 1,
                              (long long)COUT * PW))));
    ksum_kernel<<<blocks((long long)Bn * COUT * PW), 256, 0, st>>>(f->part, KSPLIT, Bn, (long long)COUT * PW, f->P);
    count_launch();
    readout_kernel<<<blocks((long long)Bn * 6 * NORD), 256, 0, st>>>(f->P, Bn, f->pred);
    count_launch();
    SC_CHECK_LAUNCH("fno forward");
    return SC_OK;
}

// gradient of sum_b loss_b / Bn into f->g (zeroed here); loss per sample into f->loss
sc_status backward(sc_fno* f, const float* tgt, int Bn, cudaStream_t st) {
    const Layout& Ly = f->lay;
    const float* w = f->w;
    float* g = f->g;
    const long long sv = (long long)W * NP, sh = (long long)HID * NP, so = (long long)COUT * NP;
    SC_CUDA_TRY(cudaMemsetAsync(g, 0, sizeof(float) * Ly.total, st));
    loss_kernel<<<Bn, 256, 0, st>>>(f->pred, tgt, Bn, f->dpred, f->loss);
    readout_back_kernel<<<blocks((long long)Bn * 6 * NORD), 256, 0, st>>>(f->dpred, Bn, f->dP);
    count_launch(2);
    // do12_b (12 x NP) = dP_b (12 x 244) R^T (the zero columns of R and dP add nothing)
    SC_TRY(gemm(st, mk(COUT, NP, PW, Bn, 1.f, 0.f, f->dP, PW, 1, (long long)COUT * PW, f->R, 1, PW, 0, f->do12, NP,
                       1, so)));
    // Q2, bQ2: per-sample partials, then summed over the batch
    SC_TRY(gemm(st, split_k(mk(COUT, HID, NP, Bn, 1.f, 0.f, f->do12, NP, 1, so, f->h, 1, NP, sh, f->part, HID, 1,
                              (long long)COUT * HID))));
    SC_TRY(batch_sum(st, f->part, Bn * KSPLIT, (long long)COUT * HID, g + Ly.Q2));
    bias_grad(st, f->do12, COUT, Bn, g + Ly.bQ2, f->bpart);
    // dh_b = Q2^T do12_b, through GELU
    SC_TRY(gemm(st, mk(HID, NP, COUT, Bn, 1.f, 0.f, w + Ly.Q2, 1, HID, 0, f->do12, NP, 1, so, f->dh, NP, 1, sh)));
    gelu_back_kernel<<<blocks((long long)Bn * sh), 256, 0, st>>>(f->dh, f->hpre, (long long)Bn * sh);
    count_launch();
    SC_TRY(gemm(st, split_k(mk(HID, W, NP, Bn, 1.f, 0.f, f->dh, NP, 1, sh, f->act[L], 1, NP, sv, f->part, W, 1,
                              (long long)HID * W))));
    SC_TRY(batch_sum(st, f->part, Bn * KSPLIT, (long long)HID * W, g + Ly.Q1));
    bias_grad(st, f->dh, HID, Bn, g + Ly.bQ1, f->bpart);
    // dv4 = Q1^T dh
    SC_TRY(gemm(st, mk(W, NP, HID, Bn, 1.f, 0.f, w + Ly.Q1, 1, W, 0, f->dh, NP, 1, sh, f->dact, NP, 1, sv)));
    for (int l = L - 1; l >= 0; --l) {
        // du = dv_{l+1} * GELU'(u_l) (no activation after the last layer)
        float* du = f->dact;
        if (l < L - 1) {
            gelu_back_kernel<<<blocks((long long)Bn * sv), 256, 0, st>>>(du, f->pre[l], (long long)Bn * sv);
            count_launch();
        }
        bias_grad(st, du, W, Bn, g + Ly.bl[l], f->bpart);
        const float* vin = f->act[l];
        // W_l
        SC_TRY(gemm(st, split_k(mk(W, W, NP, Bn, 1.f, 0.f, du, NP, 1, sv, vin, 1, NP, sv, f->part, W, 1,
                                  (long long)W * W))));
        SC_TRY(batch_sum(st, f->part, Bn * KSPLIT, (long long)W * W, g + Ly.Wl[l]));
        // dv_l = W_l^T du
        SC_TRY(gemm(st, mk(W, NP, W, Bn, 1.f, 0.f, w + Ly.Wl[l], 1, W, 0, du, NP, 1, sv, f->dv, NP, 1, sv)));
        // adjoint of the inverse transform: dZ[x][ky'][channel] = du Gy^T (batched over
        // x), dY = Er^T dZr + Ei^T dZi (mode-major)
        const long long nch = (long long)Bn * W;
        SC_TRY(gemm(st, mk((int)nch, 2 * MY, G, G, 1.f, 0.f, du, NP, 1, G, f->ops + OP_GY, 1, G, 0, f->S1, 1, nch,
                           2 * MY * nch)));
        SC_TRY(gemm(st, mk(G, (int)(MY * nch), G, 1, 1.f, 0.f, f->ops + OP_ER, 1, G, 0, f->S1, 2 * MY * nch, 1, 0, f->dY,
                           MY * nch, 1, 0)));
        SC_TRY(gemm(st, mk(G, (int)(MY * nch), G, 1, 1.f, 1.f, f->ops + OP_EI, 1, G, 0, f->S1 + MY * nch, 2 * MY * nch,
                           1, 0, f->dY, MY * nch, 1, 0)));
        // mode mixing: dX = dY M^H, dM = X^H dY (complex, per mode)
        const float* Xr = f->X[l];
        const float* Xi = f->X[l] + NM * nch;
        const float* Wr = w + Ly.SWr[l];
        const float* Wi = w + Ly.SWi[l];
        const float* dYr = f->dY;
        const float* dYi = f->dY + NM * nch;
        float* dXr = f->dX;
        float* dXi = f->dX + NM * nch;
        const long long ww = (long long)W * W;
        SC_TRY(gemm(st, mk(Bn, W, W, NM, 1.f, 0.f, dYr, W, 1, nch, Wr, 1, W, ww, dXr, W, 1, nch)));
        SC_TRY(gemm(st, mk(Bn, W, W, NM, 1.f, 1.f, dYi, W, 1, nch, Wi, 1, W, ww, dXr, W, 1, nch)));
        SC_TRY(gemm(st, mk(Bn, W, W, NM, -1.f, 0.f, dYr, W, 1, nch, Wi, 1, W, ww, dXi, W, 1, nch)));
        SC_TRY(gemm(st, mk(Bn, W, W, NM, 1.f, 1.f, dYi, W, 1, nch, Wr, 1, W, ww, dXi, W, 1, nch)));
        float* gWr = g + Ly.SWr[l];
        float* gWi = g + Ly.SWi[l];
        SC_TRY(gemm(st, mk(W, W, Bn, NM, 1.f, 0.f, Xr, 1, W, nch, dYr, W, 1, nch, gWr, W, 1, ww)));
        SC_TRY(gemm(st, mk(W, W, Bn, NM, 1.f, 1.f, Xi, 1, W, nch, dYi, W, 1, nch, gWr, W, 1, ww)));
        SC_TRY(gemm(st, mk(W, W, Bn, NM, -1.f, 0.f, Xi, 1, W, nch, dYr, W, 1, nch, gWi, W, 1, ww)));
        SC_TRY(gemm(st, mk(W, W, Bn, NM, 1.f, 1.f, Xr, 1, W, nch, dYi, W, 1, nch, gWi, W, 1, ww)));
        // adjoint of the forward transform: dU from dX, dA1 = Ex^T dU (one GEMM),
        // dv += dA1 Fy^T (batched over x)
        xcombine_back_kernel<<<blocks(nch * NM), 256, 0, st>>>(f->dX, nch, f->S2);
        count_launch();
        SC_TRY(gemm(st, mk(G, (int)(nch * 2 * MY), G, 1, 1.f, 0.f, f->ops + OP_EX, 1, G, 0, f->S2, nch * 2 * MY, 1, 0,
                           f->S1, nch * 2 * MY, 1, 0)));
        SC_TRY(gemm(st, mk((int)nch, G, 2 * MY, G, 1.f, 1.f, f->S1, 2 * MY, 1, nch * 2 * MY, f->ops + OP_FY, 1, 2 * MY,
                           0, f->dv, NP, 1, G)));
        std::swap(f->dact, f->dv);
    }
    // lift
    SC_TRY(gemm(st, split_k(mk(W, CIN, NP, Bn, 1.f, 0.f, f->dact, NP, 1, sv, f->in, 1, NP, (long long)CIN * NP, f->part,
                              CIN, 1, (long long)W * CIN))));
    SC_TRY(batch_sum(st, f->part, Bn * KSPLIT, (long long)W * CIN, g + Ly.P));
    bias_grad(st, f->dact, W, Bn, g + Ly.bP, f->bpart);
    SC_CHECK_LAUNCH("fno backward");
    return SC_OK;
}

void init_params(const Layout& Ly, uint64_t seed, std::vector<float>& w) {
    w.assign(Ly.total, 0.f);
    Rng r{seed};
    auto unif = [&](long long off, long long n, double a) {
        for (long long i = 0; i < n; ++i) w[off + i] = (float)((2.0 * r.next() - 1.0) * a);
    };
    unif(Ly.P, (long long)W * CIN, 1.0 / std::sqrt((double)CIN));
    unif(Ly.bP, W, 1.0 / std::sqrt((double)CIN));
    for (int l = 0; l < L; ++l) {
        unif(Ly.Wl[l], (long long)W * W, 1.0 / std::sqrt((double)W));
        unif(Ly.bl[l], W, 1.0 / std::sqrt((double)W));
        const double s = 1.0 / ((double)W * W);
        for (long long i = 0; i < (long long)NM * W * W; ++i) w[Ly.SWr[l] + i] = (float)(s * r.next());
        for (long long i = 0; i < (long long)NM * W * W; ++i) w[Ly.SWi[l] + i] = (float)(s * r.next());
    }
    unif(Ly.Q1, (long long)HID * W, 1.0 / std::sqrt((double)W));
    unif(Ly.bQ1, HID, 1.0 / std::sqrt((double)W));
    unif(Ly.Q2, (long long)COUT * HID, 1.0 / std::sqrt((double)HID));
    unif(Ly.bQ2, COUT, 1.0 / std::sqrt((double)HID));
}

// separable DFT operators (phases reduced mod 64 before the trigonometric call):
//   Fy (64 y x 32): [cos(2 pi ky y / 64) | -sin]                  forward along y
//   Ex (64 x 64 x): rows q < 32 cos(2 pi kx(q) x / 64), q >= 32 sin  forward along x
//   Er, Ei (64 x x 64): [cos | -sin], [sin | cos] of kx(k) x           inverse along x
//   Gy (32 x 64 y): [c cos; -c sin] / 4096, c = 1 for ky = 0 else 2   real inverse along y
// and R (NP x 244) = [cos | sin | 0 0] / NP at the 121 orders (readout)
void build_operators(std::vector<float>& ops, std::vector<float>& R) {
    ops.assign(OP_TOTAL, 0.f);
    R.assign((size_t)NP * PW, 0.f);
    const double tp = 2.0 * M_PI / G;
    auto trig = [&](long long ph, double* c, double* s) {
        const double th = tp * (double)(((ph % G) + G) % G);
        *c = std::cos(th);
        *s = std::sin(th);
    };
    double c, sn;
    for (int y = 0; y < G; ++y)
        for (int ky = 0; ky < MY; ++ky) {
            trig((long long)ky * y, &c, &sn);
            ops[OP_FY + y * 2 * MY + ky] = (float)c;
            ops[OP_FY + y * 2 * MY + MY + ky] = (float)(-sn);
            const double cw = (ky == 0 ? 1.0 : 2.0) / NP;
            ops[OP_GY + ky * G + y] = (float)(cw * c);
            ops[OP_GY + (MY + ky) * G + y] = (float)(-cw * sn);
        }
    for (int x = 0; x < G; ++x)
        for (int r = 0; r < 2 * MX; ++r) {
            trig((long long)kx_of(r) * x, &c, &sn);
            ops[OP_EX + r * G + x] = (float)c;
            ops[OP_EX + (2 * MX + r) * G + x] = (float)sn;
            ops[OP_ER + x * G + r] = (float)c;
            ops[OP_ER + x * G + 2 * MX + r] = (float)(-sn);
            ops[OP_EI + x * G + r] = (float)sn;
            ops[OP_EI + x * G + 2 * MX + r] = (float)c;
        }
    for (int x = 0; x < G; ++x)
        for (int y = 0; y < G; ++y) {
            const int p = x * G + y;
            for (int j = 0; j < NORD; ++j) {
                int pp, qq;
                order_pq(j, &pp, &qq);
                trig((long long)pp * x + (long long)qq * y, &c, &sn);
                R[(size_t)p * PW + j] = (float)(c / NP);
                R[(size_t)p * PW + NORD + j] = (float)(sn / NP);
            }
        }
}

struct Guard {
    int prev = -1;
    explicit Guard(int dev) {
        cudaGetDevice(&prev);
        cudaSetDevice(dev);
    }
    ~Guard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

sc_status check_batch(const sc_fno* f, int Bn) {
    if (!f || Bn <= 0 || Bn > f->max_batch) {
        set_error("fno: batch %d outside 1..%d", Bn, f ? f->max_batch : 0);
        return SC_BADINPUT;
    }
    return SC_OK;
}

}  // namespace

extern "C" {

sc_status sc_fno_create(sc_fno** out, int device, int max_batch, unsigned long long seed) {
    if (!out || max_batch <= 0 || max_batch > 4096) {
        set_error("sc_fno_create: bad argument (max_batch %d)", max_batch);
        return SC_BADINPUT;
    }
    *out = nullptr;
    Guard gd(device);
    sc_fno* f = new sc_fno();
    f->device = device;
    f->max_batch = max_batch;
    const Layout& Ly = f->lay;
    const long long B = max_batch, sv = (long long)W * NP;
    sc_status s = SC_OK;
    auto A = [&](float** p, long long n) {
        if (s == SC_OK) s = fno_alloc(p, n);
    };
    A(&f->w, Ly.total);
    A(&f->g, Ly.total);
    A(&f->m, Ly.total);
    A(&f->v, Ly.total);
    A(&f->ops, OP_TOTAL);
    A(&f->S1, B * W * SEP);
    A(&f->S2, B * W * SEP);
    A(&f->R, (long long)NP * PW);
    A(&f->in, B * CIN * NP);
    for (int l = 0; l <= L; ++l) A(&f->act[l], B * sv);
    for (int l = 0; l < L; ++l) {
        A(&f->pre[l], B * sv);
        A(&f->X[l], B * W * NF);
    }
    A(&f->Y, B * W * NF);
    A(&f->hpre, B * HID * NP);
    A(&f->h, B * HID * NP);
    A(&f->o12, B * COUT * NP);
    A(&f->P, B * COUT * PW);
    A(&f->pred, B * NOUT);
    A(&f->dact, B * sv);
    A(&f->dv, B * sv);
    A(&f->dX, B * W * NF);
    A(&f->dY, B * W * NF);
    A(&f->dh, B * HID * NP);
    A(&f->do12, B * COUT * NP);
    A(&f->dP, B * COUT * PW);
    A(&f->dpred, B * NOUT);
    A(&f->part, B * (long long)KSPLIT * HID * W);
    A(&f->loss, B);
    A(&f->bpart, (long long)HID * NSPL);
    if (s == SC_OK) {
        std::vector<float> w, ops, R;
        init_params(Ly, seed, w);
        build_operators(ops, R);
        cudaError_t e = cudaMemcpy(f->w, w.data(), sizeof(float) * w.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(f->ops, ops.data(), sizeof(float) * ops.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemcpy(f->R, R.data(), sizeof(float) * R.size(), cudaMemcpyHostToDevice);
        if (e == cudaSuccess) e = cudaMemset(f->m, 0, sizeof(float) * Ly.total);
        // the readout gradient's pad columns are never written: zero once
        if (e == cudaSuccess) e = cudaMemset(f->dP, 0, sizeof(float) * (size_t)B * COUT * PW);
        if (e == cudaSuccess) e = cudaMemset(f->v, 0, sizeof(float) * Ly.total);
        if (e != cudaSuccess) s = cuda_status(e, "sc_fno_create");
    }
    if (s != SC_OK) {
        sc_fno_destroy(f);
        return s;
    }
    *out = f;
    return SC_OK;
}

sc_status sc_fno_destroy(sc_fno* f) {
    if (!f) return SC_OK;
    Guard gd(f->device);
    float* ptrs[] = {f->w, f->g, f->m, f->v, f->ops, f->S1, f->S2, f->R, f->in, f->Y, f->hpre, f->h, f->o12, f->P, f->pred,
                     f->dact, f->dv, f->dX, f->dY, f->dh, f->do12, f->dP, f->dpred, f->part, f->loss, f->bpart};
    for (float* p : ptrs)
        if (p) cudaFree(p);
    for (int l = 0; l <= L; ++l)
        if (f->act[l]) cudaFree(f->act[l]);
    for (int l = 0; l < L; ++l) {
        if (f->pre[l]) cudaFree(f->pre[l]);
        if (f->X[l]) cudaFree(f->X[l]);
    }
    delete f;
    return SC_OK;
}

sc_status sc_fno_status(sc_fno* f) {
    if (!f) {
        set_error("sc_fno_status: null network");
        return SC_BADINPUT;
    }
    Guard gd(f->device);
    SC_CUDA_TRY(cudaDeviceSynchronize());
    int h = 0;
    SC_CUDA_TRY(cudaMemcpyFromSymbol(&h, g_fno_err, sizeof(int)));
    if (h) {
        const int zero = 0;
        SC_CUDA_TRY(cudaMemcpyToSymbol(g_fno_err, &zero, sizeof(int)));
        set_error("surrogate: a tensor-core GEMM pipeline wait timed out");
        return SC_CUDA_ERROR;
    }
    return SC_OK;
}

sc_status sc_fno_param_count(const sc_fno* f, long long* n) {
    if (!f || !n) {
        set_error("sc_fno_param_count: null argument");
        return SC_BADINPUT;
    }
    *n = f->lay.total;
    return SC_OK;
}

sc_status sc_fno_params(sc_fno* f, void* dev_params, int direction, void* stream) {
    if (!f || !dev_params) {
        set_error("sc_fno_params: null argument");
        return SC_BADINPUT;
    }
    Guard gd(f->device);
    const size_t bytes = sizeof(float) * (size_t)f->lay.total;
    cudaStream_t st = (cudaStream_t)stream;
    if (direction == 0)
        SC_CUDA_TRY(cudaMemcpyAsync(dev_params, f->w, bytes, cudaMemcpyDeviceToDevice, st));
    else
        SC_CUDA_TRY(cudaMemcpyAsync(f->w, dev_params, bytes, cudaMemcpyDeviceToDevice, st));
    return SC_OK;
}

sc_status sc_fno_forward(sc_fno* f, const float* maps, const float* lambdas, int batch, float* out, void* stream) {
    SC_TRY(check_batch(f, batch));
    if (!maps || !lambdas || !out) {
        set_error("sc_fno_forward: null argument");
        return SC_BADINPUT;
    }
    Guard gd(f->device);
    cudaStream_t st = (cudaStream_t)stream;
    SC_TRY(forward(f, maps, lambdas, batch, st));
    SC_CUDA_TRY(cudaMemcpyAsync(out, f->pred, sizeof(float) * (size_t)batch * NOUT, cudaMemcpyDeviceToDevice, st));
    return SC_OK;
}

sc_status sc_fno_loss_grad(sc_fno* f, const float* maps, const float* lambdas, const float* target, int batch,
                           float* loss, float* grad, void* stream) {
    SC_TRY(check_batch(f, batch));
    if (!maps || !lambdas || !target) {
        set_error("sc_fno_loss_grad: null argument");
        return SC_BADINPUT;
    }
    Guard gd(f->device);
    cudaStream_t st = (cudaStream_t)stream;
    SC_TRY(forward(f, maps, lambdas, batch, st));
    SC_TRY(backward(f, target, batch, st));
    if (loss) SC_CUDA_TRY(cudaMemcpyAsync(loss, f->loss, sizeof(float) * batch, cudaMemcpyDeviceToDevice, st));
    if (grad)
        SC_CUDA_TRY(cudaMemcpyAsync(grad, f->g, sizeof(float) * (size_t)f->lay.total, cudaMemcpyDeviceToDevice, st));
    return SC_OK;
}

sc_status sc_fno_train_step(sc_fno* f, const float* maps, const float* lambdas, const float* target, int batch,
                            float lr, float* loss, void* stream) {
    SC_TRY(sc_fno_loss_grad(f, maps, lambdas, target, batch, loss, nullptr, stream));
    cudaStream_t st = (cudaStream_t)stream;
    f->step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - std::pow(b1, (float)f->step), c2 = 1.f - std::pow(b2, (float)f->step);
    adam_kernel<<<blocks(f->lay.total), 256, 0, st>>>(f->w, f->g, f->m, f->v, f->lay.total, lr, b1, b2, 1e-8f, c1, c2);
    count_launch();
    SC_CHECK_LAUNCH("fno adam");
    return SC_OK;
}

}  // extern "C"
