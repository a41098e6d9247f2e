// Batched complex128 LU with partial pivoting (zgetrf) and the triangular
// solves that use it (zgetrs), replacing LAPACKE_zgesv behind MKL_linearsolve
// and MKL_inverse (third_Lapack.h:46-63).
//
// Right-looking blocked algorithm, NB = 32 columns per panel:
//   1. panel kernel  -- one CTA per matrix factors the n-j0 x NB panel column
//                       by column (pivot = first max |re|+|im| like izamax);
//   2. row swaps     -- applied to the columns left and right of the panel;
//   3. TRSM          -- U12 = L11^-1 A12, one thread per right-hand column;
//   4. GEMM          -- A22 -= L21 U12 through the batched zgemm tile.
// Pivots are stored 0-based as global row indices, LAPACK order.
#include "common.cuh"
#include "kernels.cuh"

namespace sc {

namespace {
constexpr int NB = 32;
constexpr int PT = 512;   // panel threads

__global__ void __launch_bounds__(PT)
panel_kernel(double2* A, int lda, long long sA, int n, int j0, int jb, int* ipiv, int* info) {
    __shared__ double red_v[PT / 32];
    __shared__ int red_i[PT / 32];
    __shared__ double2 prow[NB];
    __shared__ int s_piv;
    const int b = blockIdx.x;
    A += b * sA;
    ipiv += (long long)b * n;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    for (int jj = 0; jj < jb; ++jj) {
        const int col = j0 + jj;
        double2* c = A + (long long)col * lda;
        // pivot search
        double best = -1.0;
        int bi = n;
        for (int r = col + tid; r < n; r += PT) {
            double v = cabs1(c[r]);
            if (v > best) { best = v; bi = r; }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            double ov = __shfl_xor_sync(0xffffffffu, best, o);
            int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ov > best || (ov == best && oi < bi)) { best = ov; bi = oi; }
        }
        if (lane == 0) { red_v[wid] = best; red_i[wid] = bi; }
        __syncthreads();
        if (tid == 0) {
            double bv = -1.0;
            int bidx = n;
            for (int w = 0; w < PT / 32; ++w)
                if (red_v[w] > bv || (red_v[w] == bv && red_i[w] < bidx)) { bv = red_v[w]; bidx = red_i[w]; }
            if (bidx >= n) bidx = col;
            s_piv = bidx;
            ipiv[col] = bidx;
            if (bv == 0.0 && info != nullptr && info[b] == 0) info[b] = col + 1;
        }
        __syncthreads();
        const int p = s_piv;
        // swap rows col <-> p inside the panel
        if (p != col) {
            for (int cc = tid; cc < jb; cc += PT) {
                double2* cp = A + (long long)(j0 + cc) * lda;
                double2 t = cp[col];
                cp[col] = cp[p];
                cp[p] = t;
            }
        }
        __syncthreads();
        // pivot row (right part of the panel) to shared memory
        for (int cc = tid; cc < jb; cc += PT) prow[cc] = A[(long long)(j0 + cc) * lda + col];
        __syncthreads();
        const double2 piv = prow[jj];
        const bool nz = (piv.x != 0.0 || piv.y != 0.0);
        const double2 rp = nz ? cdiv(make_double2(1.0, 0.0), piv) : make_double2(0.0, 0.0);
        for (int r = col + 1 + tid; r < n; r += PT) {
            double2 l = nz ? cmul(c[r], rp) : c[r];
            c[r] = l;
            for (int cc = jj + 1; cc < jb; ++cc) {
                double2* cp = A + (long long)(j0 + cc) * lda + r;
                *cp = csub(*cp, cmul(l, prow[cc]));
            }
        }
        __syncthreads();
    }
}

// apply the panel's swaps ipiv[j0 .. j0+jb) to columns outside [j0, j0+jb)
__global__ void laswp_kernel(double2* A, int lda, long long sA, int n, int j0, int jb,
                             const int* ipiv, int ncols) {
    const int b = blockIdx.y;
    const int cidx = blockIdx.x * blockDim.x + threadIdx.x;
    if (cidx >= ncols) return;
    const int col = cidx < j0 ? cidx : cidx + jb;
    double2* c = A + b * sA + (long long)col * lda;
    const int* pv = ipiv + (long long)b * n;
    for (int i = j0; i < j0 + jb; ++i) {
        int p = pv[i];
        if (p != i) {
            double2 t = c[i];
            c[i] = c[p];
            c[p] = t;
        }
    }
}

// U12 = L11^-1 A12 with L11 the unit lower jb x jb block at (j0, j0)
__global__ void trsm_lunit_kernel(double2* A, int lda, long long sA, int n, int j0, int jb) {
    __shared__ double2 L[NB][NB + 1];
    const int b = blockIdx.y;
    double2* Ab = A + b * sA;
    for (int t = threadIdx.x; t < jb * jb; t += blockDim.x) {
        int i = t % jb, j = t / jb;
        L[i][j] = Ab[(long long)(j0 + j) * lda + j0 + i];
    }
    __syncthreads();
    const int col = j0 + jb + blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= n) return;
    double2 x[NB];
    double2* c = Ab + (long long)col * lda + j0;
#pragma unroll
    for (int i = 0; i < NB; ++i) x[i] = (i < jb) ? c[i] : make_double2(0.0, 0.0);
#pragma unroll
    for (int i = 1; i < NB; ++i) {
        if (i < jb) {
            double2 s = x[i];
#pragma unroll
            for (int l = 0; l < NB; ++l)
                if (l < i) s = csub(s, cmul(L[i][l], x[l]));
            x[i] = s;
        }
    }
#pragma unroll
    for (int i = 0; i < NB; ++i)
        if (i < jb) c[i] = x[i];
}

// ---------------------------------------------------------------- getrs parts
// B rows permuted by ipiv (forward order), one thread per RHS column
__global__ void laswp_rhs_kernel(double2* B, int ldb, long long sB, int n, int nrhs, const int* ipiv) {
    const int b = blockIdx.y;
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= nrhs) return;
    double2* c = B + b * sB + (long long)col * ldb;
    const int* pv = ipiv + (long long)b * n;
    for (int i = 0; i < n; ++i) {
        int p = pv[i];
        if (p != i) {
            double2 t = c[i];
            c[i] = c[p];
            c[p] = t;
        }
    }
}

// X_blk = T^-1 B_blk for the diagonal block [i0, i0+ib) of the LU factors;
// lower = unit lower (forward), else non-unit upper (backward).
template <bool LOWER>
__global__ void trsm_block_kernel(const double2* LU, int lda, long long sA, double2* B, int ldb,
                                  long long sB, int i0, int ib, int nrhs) {
    __shared__ double2 T[NB][NB + 1];
    const int b = blockIdx.y;
    const double2* Ab = LU + b * sA;
    for (int t = threadIdx.x; t < ib * ib; t += blockDim.x) {
        int i = t % ib, j = t / ib;
        T[i][j] = Ab[(long long)(i0 + j) * lda + i0 + i];
    }
    __syncthreads();
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= nrhs) return;
    double2* c = B + b * sB + (long long)col * ldb + i0;
    double2 x[NB];
#pragma unroll
    for (int i = 0; i < NB; ++i) x[i] = (i < ib) ? c[i] : make_double2(0.0, 0.0);
    if (LOWER) {
#pragma unroll
        for (int i = 1; i < NB; ++i) {
            if (i < ib) {
                double2 s = x[i];
#pragma unroll
                for (int l = 0; l < NB; ++l)
                    if (l < i) s = csub(s, cmul(T[i][l], x[l]));
                x[i] = s;
            }
        }
    } else {
#pragma unroll
        for (int i = NB - 1; i >= 0; --i) {
            if (i < ib) {
                double2 s = x[i];
#pragma unroll
                for (int l = 0; l < NB; ++l)
                    if (l > i && l < ib) s = csub(s, cmul(T[i][l], x[l]));
                double2 d = T[i][i];
                x[i] = (d.x != 0.0 || d.y != 0.0) ? cdiv(s, d) : s;
            }
        }
    }
#pragma unroll
    for (int i = 0; i < NB; ++i)
        if (i < ib) c[i] = x[i];
}

__global__ void set_identity_kernel(double2* B, int ldb, long long sB, int n) {
    const int b = blockIdx.y;
    long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)n * n) return;
    int i = (int)(t % n), j = (int)(t / n);
    B[b * sB + (long long)j * ldb + i] = make_double2(i == j ? 1.0 : 0.0, 0.0);
}
}  // namespace

sc_status getrf(cudaStream_t st, double2* A, int lda, long long sA, int n, int batch, int* ipiv,
                int* info) {
    if (n <= 0 || batch <= 0) return SC_OK;
    if (batch > 65535) {
        set_error("getrf: batch %d too large", batch);
        return SC_BADINPUT;
    }
    for (int j0 = 0; j0 < n; j0 += NB) {
        const int jb = (n - j0) < NB ? (n - j0) : NB;
        panel_kernel<<<batch, PT, 0, st>>>(A, lda, sA, n, j0, jb, ipiv, info);
        count_launch();
        const int ncols = n - jb;
        if (ncols > 0) {
            dim3 g((ncols + 127) / 128, batch);
            laswp_kernel<<<g, 128, 0, st>>>(A, lda, sA, n, j0, jb, ipiv, ncols);
            count_launch();
        }
        const int rest = n - j0 - jb;
        if (rest > 0) {
            dim3 g((rest + 127) / 128, batch);
            trsm_lunit_kernel<<<g, 128, 0, st>>>(A, lda, sA, n, j0, jb);
            count_launch();
            SC_TRY(zgemm(st, rest, rest, jb, make_double2(-1.0, 0.0),
                         A + (long long)j0 * lda + j0 + jb, lda, sA,
                         A + (long long)(j0 + jb) * lda + j0, lda, sA, make_double2(1.0, 0.0),
                         A + (long long)(j0 + jb) * lda + j0 + jb, lda, sA, batch));
        }
    }
    SC_CHECK_LAUNCH("getrf");
    return SC_OK;
}

sc_status getrs(cudaStream_t st, const double2* LU, int lda, long long sA, int n, const int* ipiv,
                double2* B, int ldb, long long sB, int nrhs, int batch) {
    if (n <= 0 || nrhs <= 0 || batch <= 0) return SC_OK;
    const int tpb = 64;
    dim3 g((nrhs + tpb - 1) / tpb, batch);
    laswp_rhs_kernel<<<g, tpb, 0, st>>>(B, ldb, sB, n, nrhs, ipiv);
    count_launch();
    // forward: L y = b
    for (int i0 = 0; i0 < n; i0 += NB) {
        const int ib = (n - i0) < NB ? (n - i0) : NB;
        trsm_block_kernel<true><<<g, tpb, 0, st>>>(LU, lda, sA, B, ldb, sB, i0, ib, nrhs);
        count_launch();
        const int rest = n - i0 - ib;
        if (rest > 0)
            SC_TRY(zgemm(st, rest, nrhs, ib, make_double2(-1.0, 0.0), LU + (long long)i0 * lda + i0 + ib,
                         lda, sA, B + i0, ldb, sB, make_double2(1.0, 0.0), B + i0 + ib, ldb, sB, batch));
    }
    // backward: U x = y
    const int nblk = (n + NB - 1) / NB;
    for (int bi = nblk - 1; bi >= 0; --bi) {
        const int i0 = bi * NB;
        const int ib = (n - i0) < NB ? (n - i0) : NB;
        trsm_block_kernel<false><<<g, tpb, 0, st>>>(LU, lda, sA, B, ldb, sB, i0, ib, nrhs);
        count_launch();
        if (i0 > 0)
            SC_TRY(zgemm(st, i0, nrhs, ib, make_double2(-1.0, 0.0), LU + (long long)i0 * lda, lda, sA,
                         B + i0, ldb, sB, make_double2(1.0, 0.0), B, ldb, sB, batch));
    }
    SC_CHECK_LAUNCH("getrs");
    return SC_OK;
}

sc_status set_identity(cudaStream_t st, double2* B, int ldb, long long sB, int n, int batch) {
    long long tot = (long long)n * n;
    dim3 g((unsigned)((tot + 255) / 256), batch);
    set_identity_kernel<<<g, 256, 0, st>>>(B, ldb, sB, n);
    count_launch();
    SC_CHECK_LAUNCH("set_identity");
    return SC_OK;
}

}  // namespace sc
