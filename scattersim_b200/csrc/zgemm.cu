// Batched complex128 GEMM, C = alpha * op(A) * op(B) + beta * C (column-major,
// op = identity or conjugate transpose).
//
// Replaces cblas_zgemm behind MKL_multiply (third_Lapack.h:74-84) and every
// dense product of the layer chain, the boundary system and the interior
// fields (ScatterVolume.cpp:331-334, 447-449, 769-779, 838-839).
//
// The tile runs on the FP64 tensor pipe (mma.sync m8n8k4 f64, measured 37.1
// TFLOP/s against 36.6 for DFMA): a complex 8 x 8 x 4 product is four real
// MMAs (Re += Ar Br - Ai Bi, Im += Ar Bi + Ai Br), so operand reuse happens
// inside the MMA unit and shared memory feeds one complex fragment value per
// lane per MMA group instead of a full outer product per thread.  256 threads
// (8 warps) per CTA; each warp owns MT x NT 8 x 8 complex tiles.  Two CTA
// shapes: 128 x 64 (warps 4 x 2, 32 x 32 each) for large products and 64 x 64
// (warps 2 x 4, 32 x 16 each, two CTAs per SM) for short K or when the large
// tile would leave SMs idle.  K is
// staged 16 deep through a three-stage cp.async ring (16-byte copies,
// zero-filled past the edges); op = ^H is applied to fragments as they leave
// shared memory.
#include "common.cuh"
#include "kernels.cuh"

namespace sc {

namespace {
constexpr int BK = 16, NT = 256, ST = 3;

__device__ __forceinline__ void cp16(void* smem, const void* gmem, bool pred) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    const int n = pred ? 16 : 0;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(n));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

template <int BM>
constexpr int tile_smem_bytes() {
    return ST * BK * ((BM + 1) + (64 + 1)) * (int)sizeof(double2);
}

// d (8x8, two values per lane) += a (8x4 row fragment) * b (4x8 column fragment)
__device__ __forceinline__ void dmma(double* d, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// CA / CB: operand is used conjugate-transposed (op = ^H) instead of as is
template <int BM, bool CA, bool CB>
__global__ void __launch_bounds__(NT, (BM == 64 ? 2 : 1)) zgemm_kernel(GemmArgs g) {
    constexpr int BN = 64;
    constexpr int WM = (BM == 128) ? 4 : 2, WN = 8 / WM;     // warps along m, n
    constexpr int MT = BM / WM / 8, NT8 = BN / WN / 8;       // 8x8 tiles per warp
    constexpr int LAS = BM + 1, LBS = BN + 1;
    extern __shared__ double2 smem[];
    double2* As = smem;                    // [ST][BK][LAS]
    double2* Bs = smem + ST * BK * LAS;    // [ST][BK][LBS]
    const int bz = blockIdx.z;
    const int m = g.m, n = g.n, k = g.k, lda = g.lda, ldb = g.ldb, ldc = g.ldc;
    // per-CTA operand addresses: pointer arrays when given, else strided
    const double2* __restrict__ A = g.Ap ? g.Ap[bz] : g.A + bz * g.sA;
    const double2* __restrict__ B = g.Bp ? g.Bp[bz] : g.B + bz * g.sB;
    double2* __restrict__ C = g.Cp ? g.Cp[bz] : g.C + bz * g.sC;
    const double2 alpha = g.alphas ? cmul(g.alpha, g.alphas[bz]) : g.alpha;
    const double2 beta = g.beta;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp % WM, wn = warp / WM;
    const int gq = lane >> 2, tq = lane & 3;   // fragment row/col group, thread in group

    // consecutive threads copy consecutive global addresses
    auto load_stage = [&](int slot, int k0) {
        double2* as = As + slot * BK * LAS;
        double2* bs = Bs + slot * BK * LBS;
#pragma unroll
        for (int i = 0; i < BM * BK / NT; ++i) {
            const int e = tid + NT * i;
            int r, kk;
            if (!CA) { r = e % BM; kk = e / BM; }
            else { kk = e % BK; r = e / BK; }
            const int gr = m0 + r, gk = k0 + kk;
            const bool ok = gr < m && gk < k;
            const double2* src = ok ? (CA ? A + (long long)gr * lda + gk : A + (long long)gk * lda + gr) : A;
            cp16(as + kk * LAS + r, src, ok);
        }
#pragma unroll
        for (int i = 0; i < BN * BK / NT; ++i) {
            const int e = tid + NT * i;
            int kk, c;
            if (!CB) { kk = e % BK; c = e / BK; }
            else { c = e % BN; kk = e / BN; }
            const int gk = k0 + kk, gc = n0 + c;
            const bool ok = gk < k && gc < n;
            const double2* src = ok ? (CB ? B + (long long)gk * ldb + gc : B + (long long)gc * ldb + gk) : B;
            cp16(bs + kk * LBS + c, src, ok);
        }
    };

    double cr[MT][NT8][2], ci[MT][NT8][2];
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT8; ++j) cr[i][j][0] = cr[i][j][1] = ci[i][j][0] = ci[i][j][1] = 0.0;

    const int nk = (k + BK - 1) / BK;
#pragma unroll
    for (int s = 0; s < ST - 1; ++s) {
        if (s < nk) load_stage(s, s * BK);
        cp_commit();
    }
    const int arow = wm * MT * 8 + gq;   // + 8 * mt
    const int bcol = wn * NT8 * 8 + gq;  // + 8 * nt
    for (int t = 0; t < nk; ++t) {
        cp_wait<ST - 2>();
        __syncthreads();
        const int tn = t + ST - 1;
        if (tn < nk) load_stage(tn % ST, tn * BK);
        cp_commit();
        const double2* as = As + (t % ST) * BK * LAS;
        const double2* bs = Bs + (t % ST) * BK * LBS;
#pragma unroll
        for (int ks = 0; ks < BK; ks += 4) {
            double2 a[MT], b[NT8];
#pragma unroll
            for (int i = 0; i < MT; ++i) {
                a[i] = as[(ks + tq) * LAS + arow + 8 * i];
                if (CA) a[i].y = -a[i].y;
            }
#pragma unroll
            for (int j = 0; j < NT8; ++j) {
                b[j] = bs[(ks + tq) * LBS + bcol + 8 * j];
                if (CB) b[j].y = -b[j].y;
            }
#pragma unroll
            for (int i = 0; i < MT; ++i)
#pragma unroll
                for (int j = 0; j < NT8; ++j) {
                    dmma(cr[i][j], a[i].x, b[j].x);
                    dmma(ci[i][j], a[i].x, b[j].y);
                    dmma(ci[i][j], a[i].y, b[j].x);
                    dmma(cr[i][j], -a[i].y, b[j].y);
                }
        }
    }
    cp_wait<0>();
    const bool beta_zero = (beta.x == 0.0 && beta.y == 0.0);
#pragma unroll
    for (int i = 0; i < MT; ++i) {
        const int gr = m0 + arow + 8 * i;
        if (gr >= m) continue;
#pragma unroll
        for (int j = 0; j < NT8; ++j) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int gc = n0 + wn * NT8 * 8 + 8 * j + 2 * tq + h;
                if (gc >= n) continue;
                double2* p = C + (long long)gc * ldc + gr;
                double2 v = cmul(alpha, make_double2(cr[i][j][h], ci[i][j][h]));
                if (!beta_zero) v = cfma(beta, *p, v);
                *p = v;
            }
        }
    }
}

template <int BM, bool CA, bool CB>
sc_status launch_tile(cudaStream_t st, const GemmArgs& g, int batch) {
    constexpr int bytes = tile_smem_bytes<BM>();
    SC_TRY(smem_opt_in(zgemm_kernel<BM, CA, CB>, bytes));
    dim3 grid((g.m + BM - 1) / BM, (g.n + 63) / 64, batch);
    zgemm_kernel<BM, CA, CB><<<grid, NT, bytes, st>>>(g);
    return SC_OK;
}

template <int BM>
sc_status launch_shape(cudaStream_t st, bool conjA, bool conjB, const GemmArgs& g, int batch) {
    if (!conjA && !conjB) return launch_tile<BM, false, false>(st, g, batch);
    if (conjA && !conjB) return launch_tile<BM, true, false>(st, g, batch);
    if (!conjA && conjB) return launch_tile<BM, false, true>(st, g, batch);
    return launch_tile<BM, true, true>(st, g, batch);
}
}  // namespace

sc_status zgemm_tile(cudaStream_t st, bool conjA, bool conjB, const GemmArgs& g, int batch, int tile) {
    if (g.m <= 0 || g.n <= 0 || batch <= 0) return SC_OK;
    if ((g.n + 63) / 64 > 65535 || batch > 65535) {
        set_error("zgemm: grid too large (n=%d, batch=%d)", g.n, batch);
        return SC_BADINPUT;
    }
    if (tile == 128)
        SC_TRY(launch_shape<128>(st, conjA, conjB, g, batch));
    else
        SC_TRY(launch_shape<64>(st, conjA, conjB, g, batch));
    count_launch();
    SC_CHECK_LAUNCH("zgemm");
    return SC_OK;
}

sc_status zgemm_run(cudaStream_t st, bool conjA, bool conjB, const GemmArgs& g, int batch) {
    // the 128-row tile when it still gives every SM at least one CTA and K is
    // deep enough to amortise its pipeline fill (rank-32 panel updates of the
    // LU and Hessenberg reductions stay on the two-CTA-per-SM 64-row tile)
    const long long big = (long long)((g.m + 127) / 128) * ((g.n + 63) / 64) * batch;
    const int tile = (g.m > 64 && g.k > 48 && big >= 148) ? 128 : 64;
    return zgemm_tile(st, conjA, conjB, g, batch, tile);
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
