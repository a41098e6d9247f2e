// Batched complex128 GEMM, C = alpha * op(A) * op(B) + beta * C (column-major,
// op = identity or conjugate transpose).
//
// Replaces cblas_zgemm behind MKL_multiply (third_Lapack.h:74-84) and every
// dense product of the layer chain, the boundary system and the interior
// fields (ScatterVolume.cpp:331-334, 447-449, 769-779, 838-839).
//
// FP64 throughput on B200 is the same through DFMA and DMMA, so the tile is a
// register-blocked SIMT DFMA tile: 64 x 64 complex outputs per CTA of 256
// threads, each thread owning a 4 x 4 complex block strided by 16 so that
// shared-memory reads and global stores are contiguous across a warp.  The
// K dimension is staged through shared memory 16 deep; the next tile's global
// loads are issued into registers before the current tile's math.
#include "common.cuh"
#include "kernels.cuh"

namespace sc {

namespace {
constexpr int BM = 64, BN = 64, BK = 16, NT = 256;

// CA / CB: operand is used conjugate-transposed (op = ^H) instead of as is
template <bool CA, bool CB>
__global__ void __launch_bounds__(NT, 2) zgemm_kernel(GemmArgs g) {
    __shared__ double2 As[BK][BM];
    __shared__ double2 Bs[BK][BN + 1];
    const int bz = blockIdx.z;
    const int m = g.m, n = g.n, k = g.k, lda = g.lda, ldb = g.ldb, ldc = g.ldc;
    // per-CTA operand addresses: pointer arrays when given, else strided
    const double2* __restrict__ A = g.Ap ? g.Ap[bz] : g.A + bz * g.sA;
    const double2* __restrict__ B = g.Bp ? g.Bp[bz] : g.B + bz * g.sB;
    double2* __restrict__ C = g.Cp ? g.Cp[bz] : g.C + bz * g.sC;
    const double2 alpha = g.alphas ? cmul(g.alpha, g.alphas[bz]) : g.alpha;
    const double2 beta = g.beta;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;

    // global -> register staging: A tile 64x16 (4 per thread), B tile 16x64 (4 per thread)
    double2 ra[4], rb[4];
    // index maps chosen so that consecutive threads read consecutive addresses
    auto a_rk = [&](int i, int& r, int& kk) {
        if (!CA) { r = tid & 63; kk = (tid >> 6) + 4 * i; }
        else { r = (tid >> 4) + 16 * i; kk = tid & 15; }
    };
    auto b_kc = [&](int i, int& kk, int& c) {
        if (!CB) { kk = tid & 15; c = (tid >> 4) + 16 * i; }
        else { kk = (tid >> 6) + 4 * i; c = tid & 63; }
    };
    auto load = [&](int k0) {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            int r, kk;
            a_rk(i, r, kk);
            int gr = m0 + r, gk = k0 + kk;
            if (gr < m && gk < k)
                ra[i] = CA ? cconj(A[(long long)gr * lda + gk]) : A[(long long)gk * lda + gr];
            else
                ra[i] = make_double2(0.0, 0.0);
            int kb, c;
            b_kc(i, kb, c);
            int gkb = k0 + kb, gc = n0 + c;
            if (gkb < k && gc < n)
                rb[i] = CB ? cconj(B[(long long)gkb * ldb + gc]) : B[(long long)gc * ldb + gkb];
            else
                rb[i] = make_double2(0.0, 0.0);
        }
    };
    auto store = [&]() {
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            int r, kk, kb, c;
            a_rk(i, r, kk);
            b_kc(i, kb, c);
            As[kk][r] = ra[i];
            Bs[kb][c] = rb[i];
        }
    };

    double2 acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = make_double2(0.0, 0.0);

    int nk = (k + BK - 1) / BK;
    if (nk > 0) {
        load(0);
        store();
    }
    __syncthreads();
    for (int t = 0; t < nk; ++t) {
        if (t + 1 < nk) load((t + 1) * BK);
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            double2 a[4], b[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) a[i] = As[kk][tx + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = Bs[kk][ty + 16 * j];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) acc[i][j] = cfma(a[i], b[j], acc[i][j]);
        }
        __syncthreads();
        if (t + 1 < nk) {
            store();
            __syncthreads();
        }
    }
    const bool beta_zero = (beta.x == 0.0 && beta.y == 0.0);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        int gc = n0 + ty + 16 * j;
        if (gc >= n) continue;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            int gr = m0 + tx + 16 * i;
            if (gr >= m) continue;
            double2* p = C + (long long)gc * ldc + gr;
            double2 v = cmul(alpha, acc[i][j]);
            if (!beta_zero) v = cfma(beta, *p, v);
            *p = v;
        }
    }
}
}  // namespace

sc_status zgemm_run(cudaStream_t st, bool conjA, bool conjB, const GemmArgs& g, int batch) {
    if (g.m <= 0 || g.n <= 0 || batch <= 0) return SC_OK;
    dim3 grid((g.m + BM - 1) / BM, (g.n + BN - 1) / BN, batch);
    if (grid.y > 65535 || grid.z > 65535) {
        set_error("zgemm: grid too large (n=%d, batch=%d)", g.n, batch);
        return SC_BADINPUT;
    }
    if (!conjA && !conjB)
        zgemm_kernel<false, false><<<grid, NT, 0, st>>>(g);
    else if (conjA && !conjB)
        zgemm_kernel<true, false><<<grid, NT, 0, st>>>(g);
    else if (!conjA && conjB)
        zgemm_kernel<false, true><<<grid, NT, 0, st>>>(g);
    else
        zgemm_kernel<true, true><<<grid, NT, 0, st>>>(g);
    count_launch();
    SC_CHECK_LAUNCH("zgemm");
    return SC_OK;
}

sc_status zgemm_op(cudaStream_t st, bool conjA, bool conjB, int m, int n, int k, double2 alpha,
                   const double2* A, int lda, long long sA, const double2* B, int ldb, long long sB,
                   double2 beta, double2* C, int ldc, long long sC, int batch) {
    GemmArgs g;
    g.m = m;
    g.n = n;
    g.k = k;
    g.alpha = alpha;
    g.beta = beta;
    g.A = A;
    g.lda = lda;
    g.sA = sA;
    g.B = B;
    g.ldb = ldb;
    g.sB = sB;
    g.C = C;
    g.ldc = ldc;
    g.sC = sC;
    return zgemm_run(st, conjA, conjB, g, batch);
}

namespace {
constexpr int VR = 128;   // rows per GEMV CTA
constexpr int VC = 64;    // columns per GEMV partial

// part[b][ch][r] = sum over columns of chunk ch of A[r, c] x[c]
__global__ void __launch_bounds__(VR)
zgemv_part_kernel(int m, int n, const double2* __restrict__ A, int lda, long long sA,
                  const double2* __restrict__ x, long long sx, double2* __restrict__ part, int nch) {
    __shared__ double2 xs[VC];
    const int b = blockIdx.z, ch = blockIdx.x;
    const int c0 = ch * VC, c1 = (c0 + VC < n) ? c0 + VC : n;
    for (int q = threadIdx.x; q < c1 - c0; q += VR) xs[q] = x[b * sx + c0 + q];
    __syncthreads();
    const int r = blockIdx.y * VR + threadIdx.x;
    if (r >= m) return;
    const double2* a = A + b * sA + (long long)c0 * lda + r;
    double2 acc = make_double2(0.0, 0.0);
#pragma unroll 8
    for (int q = 0; q < c1 - c0; ++q) acc = cfma(a[(long long)q * lda], xs[q], acc);
    part[((long long)b * nch + ch) * m + r] = acc;
}

// y = alpha * sum_ch part + beta * y (fixed summation order)
__global__ void zgemv_sum_kernel(int m, const double2* __restrict__ part, int nch, double2 alpha, double2 beta,
                                 double2* __restrict__ y, long long sy) {
    const int b = blockIdx.y;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= m) return;
    double2 acc = make_double2(0.0, 0.0);
    for (int ch = 0; ch < nch; ++ch) acc = cadd(acc, part[((long long)b * nch + ch) * m + r]);
    double2 v = cmul(alpha, acc);
    if (beta.x != 0.0 || beta.y != 0.0) v = cfma(beta, y[b * sy + r], v);
    y[b * sy + r] = v;
}
}  // namespace

sc_status zgemv(cudaStream_t st, int m, int n, double2 alpha, const double2* A, int lda, long long sA,
                const double2* x, long long sx, double2 beta, double2* y, long long sy, int batch, double2* part) {
    if (m <= 0 || batch <= 0) return SC_OK;
    const int nch = (n + VC - 1) / VC;
    if (nch == 0) return SC_OK;
    dim3 g(nch, (m + VR - 1) / VR, batch);
    zgemv_part_kernel<<<g, VR, 0, st>>>(m, n, A, lda, sA, x, sx, part, nch);
    count_launch();
    dim3 g2((m + 255) / 256, batch);
    zgemv_sum_kernel<<<g2, 256, 0, st>>>(m, part, nch, alpha, beta, y, sy);
    count_launch();
    SC_CHECK_LAUNCH("zgemv");
    return SC_OK;
}

size_t zgemv_part_size(int m, int n, int batch) { return (size_t)batch * ((n + VC - 1) / VC) * m; }

sc_status zgemm(cudaStream_t st, int m, int n, int k, double2 alpha, const double2* A, int lda,
                long long sA, const double2* B, int ldb, long long sB, double2 beta, double2* C,
                int ldc, long long sC, int batch) {
    return zgemm_op(st, false, false, m, n, k, alpha, A, lda, sA, B, ldb, sB, beta, C, ldc, sC, batch);
}

}  // namespace sc
