// Blocked Householder reduction to upper Hessenberg form and the explicit
// unitary Q, for a batch of n x n complex128 matrices (the work of zgehrd +
// zunghr inside LAPACKE_zgeev, third_Lapack.h:37-44).
//
// Panels of NBH = 32 columns (the zlahr2 formulation).  With the reflectors
// H_l = I - tau_l v_l v_l^H of the current panel accumulated as
// P_j = H_0 ... H_{j-1} = I - V_j T_j V_j^H and Y_j = A V_j T_j (A = matrix at
// the start of the panel), column c = k + j of P_j^H A P_j is
//     x = A[:, c] - Y_j conj(V_j[c, :]);  x[k+1:] -= V_j T_j^H V_j^H x[k+1:]
// and the next column of Y is  y_j = tau_j (A v_j - Y_j (V_j^H v_j)).
// Per reflector: one CTA per matrix forms the column and the reflector
// (col_kernel), and a multi-CTA GEMV computes A v_j over the trailing columns
// for all matrices at once (gemv_kernel, deterministic two-pass reduction).
// After each panel the trailing matrix gets  A -= Y V^H  (right) and
// A <- (I - V T^H V^H) A  (left) as batched GEMMs.  Q is accumulated panel by
// panel from the last one, Q <- (I - V T V^H) Q, also as GEMMs.
#include "common.cuh"
#include "kernels.cuh"

namespace sc {

namespace {
constexpr int NBH = 32;   // panel width
constexpr int CT = 512;   // column kernel threads
constexpr int GCH = 64;   // columns per GEMV partial
constexpr int GR = 128;   // rows per GEMV CTA

struct HessPtrs {
    double2* A;      // n x n, stride n*n
    double2* Y;      // n x NBH, stride n*NBH
    double2* V;      // n x NBH, stride n*NBH
    double2* T;      // npan x NBH x NBH, stride sT
    double2* tau;    // n, stride n
    double2* part;   // nchmax x n, stride nchmax*n
    double2* wv;     // NBH, stride NBH
    long long sT;
    int nchmax;
};

// j < ib: finalise y_{j-1}, then form column k+j and reflector j.
// j == ib: only finalise y_{ib-1}.
__global__ void __launch_bounds__(CT)
col_kernel(HessPtrs P, int n, int k, int j, int ib, int panel, int nch_prev) {
    extern __shared__ double2 x[];          // n
    __shared__ double2 vc[NBH], t[NBH], t2[NBH], wl[NBH];
    __shared__ double red[32];
    __shared__ double2 s_tau, s_scal;
    __shared__ double s_beta;
    const int b = blockIdx.x, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int nw = CT / 32;
    double2* A = P.A + (long long)b * n * n;
    double2* Y = P.Y + (long long)b * n * NBH;
    double2* V = P.V + (long long)b * n * NBH;
    double2* T = P.T + (long long)b * P.sT + (long long)panel * NBH * NBH;
    double2* tau = P.tau + (long long)b * n;
    const double2* part = P.part + (long long)b * P.nchmax * n;
    double2* wv = P.wv + (long long)b * NBH;
    if (j == 0) {
        for (int q = tid; q < NBH * NBH; q += CT) T[q] = make_double2(0.0, 0.0);
    }
    // ---- finalise y_{j-1} = tau (A v - Y_{j-1} w)
    if (j > 0) {
        const double2 tp = tau[k + j - 1];
        if (tid < j - 1) wl[tid] = wv[tid];
        __syncthreads();
        for (int r = tid; r < n; r += CT) {
            double2 u = make_double2(0.0, 0.0);
            for (int ch = 0; ch < nch_prev; ++ch) u = cadd(u, part[(long long)ch * n + r]);
            for (int l = 0; l < j - 1; ++l) u = csub(u, cmul(Y[(long long)l * n + r], wl[l]));
            Y[(long long)(j - 1) * n + r] = cmul(tp, u);
        }
        __syncthreads();
    }
    if (j >= ib) return;
    const int c = k + j;
    // ---- x = A[:, c] - Y_j conj(V_j[c, :])
    if (tid < j) vc[tid] = V[(long long)tid * n + c];
    __syncthreads();
    for (int r = tid; r < n; r += CT) {
        double2 v = A[(long long)c * n + r];
        for (int l = 0; l < j; ++l) v = csub(v, cmulc(Y[(long long)l * n + r], vc[l]));
        x[r] = v;
    }
    __syncthreads();
    // ---- x[k+1:] -= V_j T_j^H (V_j^H x[k+1:])
    if (j > 0) {
        for (int l = wid; l < j; l += nw) {
            double2 acc = make_double2(0.0, 0.0);
            const double2* vl = V + (long long)l * n;
            for (int r = k + 1 + lane; r < n; r += 32) acc = cfma(cconj(vl[r]), x[r], acc);
            acc = warp_sum2(acc);
            if (lane == 0) t[l] = acc;
        }
        __syncthreads();
        if (tid < j) {
            double2 acc = make_double2(0.0, 0.0);
            for (int l2 = 0; l2 <= tid; ++l2) acc = cfma(cconj(T[(long long)tid * NBH + l2]), t[l2], acc);
            t2[tid] = acc;
        }
        __syncthreads();
        for (int r = k + 1 + tid; r < n; r += CT) {
            double2 v = x[r];
            for (int l = 0; l < j; ++l) v = csub(v, cmul(V[(long long)l * n + r], t2[l]));
            x[r] = v;
        }
        __syncthreads();
    }
    // ---- reflector from x[k+1+j:]
    const int r0 = k + 1 + j;
    double loc = 0.0;
    for (int r = r0 + 1 + tid; r < n; r += CT) loc += cnorm2(x[r]);
    const double xn2 = block_sum(loc, red);
    if (tid == 0) {
        const double2 alpha = x[r0];
        if (xn2 == 0.0 && alpha.y == 0.0) {
            s_tau = make_double2(0.0, 0.0);
            s_scal = make_double2(1.0, 0.0);
            s_beta = alpha.x;
        } else {
            const double beta = -copysign(sqrt(alpha.x * alpha.x + alpha.y * alpha.y + xn2), alpha.x);
            s_tau = make_double2((beta - alpha.x) / beta, -alpha.y / beta);
            s_scal = cdiv(make_double2(1.0, 0.0), make_double2(alpha.x - beta, alpha.y));
            s_beta = beta;
        }
    }
    __syncthreads();
    const double2 tv = s_tau, scal = s_scal;
    double2* vj = V + (long long)j * n;
    for (int r = tid; r < n; r += CT) {
        double2 xv = x[r], vv;
        if (r < r0) {
            vv = make_double2(0.0, 0.0);
        } else if (r == r0) {
            vv = make_double2(1.0, 0.0);
            xv = make_double2(s_beta, 0.0);
        } else {
            xv = cmul(xv, scal);
            vv = xv;
        }
        A[(long long)c * n + r] = xv;
        vj[r] = vv;
    }
    if (tid == 0) tau[c] = tv;
    __syncthreads();
    // ---- w = V_j^H v_j ; T[:, j] = -tau T_j w, T[j, j] = tau
    for (int l = wid; l < j; l += nw) {
        double2 acc = make_double2(0.0, 0.0);
        const double2* vl = V + (long long)l * n;
        for (int r = r0 + lane; r < n; r += 32) acc = cfma(cconj(vl[r]), vj[r], acc);
        acc = warp_sum2(acc);
        if (lane == 0) wl[l] = acc;
    }
    __syncthreads();
    if (tid < j) {
        wv[tid] = wl[tid];
        double2 acc = make_double2(0.0, 0.0);
        for (int l2 = tid; l2 < j; ++l2) acc = cfma(T[(long long)l2 * NBH + tid], wl[l2], acc);
        T[(long long)j * NBH + tid] = cneg(cmul(tv, acc));
    }
    if (tid == 0) T[(long long)j * NBH + j] = tv;
}

// part[ch][r] = sum over the chunk's columns c >= c0 of A[r, c] v[c], v = V[:, j]
__global__ void __launch_bounds__(GR)
gemv_kernel(HessPtrs P, int n, int c0, int j) {
    __shared__ double2 vs[GCH];
    const int b = blockIdx.z, ch = blockIdx.x;
    const int cbeg = c0 + ch * GCH;
    const int cend = (cbeg + GCH < n) ? cbeg + GCH : n;
    const double2* A = P.A + (long long)b * n * n;
    const double2* v = P.V + (long long)b * n * NBH + (long long)j * n;
    for (int q = threadIdx.x; q < cend - cbeg; q += GR) vs[q] = v[cbeg + q];
    __syncthreads();
    const int r = blockIdx.y * GR + threadIdx.x;
    if (r >= n) return;
    double2 acc = make_double2(0.0, 0.0);
    const double2* a = A + (long long)cbeg * n + r;
#pragma unroll 8
    for (int q = 0; q < cend - cbeg; ++q) acc = cfma(a[(long long)q * n], vs[q], acc);
    P.part[(long long)b * P.nchmax * n + (long long)ch * n + r] = acc;
}

// V of panel (k, ib) rebuilt from the reflectors stored below A's subdiagonal
__global__ void panel_v_kernel(const double2* Aall, int n, int k, int ib, double2* Vall) {
    const int b = blockIdx.y;
    const double2* A = Aall + (long long)b * n * n;
    double2* V = Vall + (long long)b * n * NBH;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < (long long)n * ib;
         q += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(q % n), l = (int)(q / n);
        const int r0 = k + 1 + l;
        V[(long long)l * n + r] = (r < r0) ? make_double2(0.0, 0.0)
                                : (r == r0) ? make_double2(1.0, 0.0) : A[(long long)(k + l) * n + r];
    }
}

__global__ void identity_clear_kernel(double2* Qall, double2* Aall, int n) {
    const int b = blockIdx.y;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < (long long)n * n;
         q += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(q % n), c = (int)(q / n);
        Qall[(long long)b * n * n + q] = make_double2(r == c ? 1.0 : 0.0, 0.0);
        (void)Aall;
    }
}

__global__ void clear_below_kernel(double2* Aall, int n) {
    const int b = blockIdx.y;
    for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < (long long)n * n;
         q += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(q % n), c = (int)(q / n);
        if (r > c + 1) Aall[(long long)b * n * n + q] = make_double2(0.0, 0.0);
    }
}

unsigned gridfor(long long tot) {
    long long g = (tot + 255) / 256;
    if (g > 4096) g = 4096;
    if (g < 1) g = 1;
    return (unsigned)g;
}
}  // namespace

sc_status hessenberg_blocked(cudaStream_t st, double2* A, int n, int batch, double2* Q, Workspace& ws) {
    if (n <= 0 || batch <= 0) return SC_OK;
    const int npan = (n - 1 + NBH - 1) / NBH;
    const int nchmax = (n + GCH - 1) / GCH;
    HessPtrs P;
    P.A = A;
    P.sT = (long long)(npan > 0 ? npan : 1) * NBH * NBH;
    P.nchmax = nchmax;
    SC_TRY(ws.get(&P.Y, (size_t)batch * n * NBH, WS_HY, st));
    SC_TRY(ws.get(&P.V, (size_t)batch * n * NBH, WS_HV, st));
    SC_TRY(ws.get(&P.T, (size_t)batch * P.sT, WS_HT, st));
    SC_TRY(ws.get(&P.part, (size_t)batch * nchmax * n, WS_HPART, st));
    SC_TRY(ws.get(&P.tau, (size_t)batch * n + (size_t)batch * NBH, WS_EIG_TAU, st));
    P.wv = P.tau + (size_t)batch * n;
    double2 *W, *W2;
    SC_TRY(ws.get(&W, (size_t)batch * NBH * n, WS_HW, st));
    SC_TRY(ws.get(&W2, (size_t)batch * NBH * n, WS_HW2, st));
    const size_t xsm = (size_t)n * sizeof(double2);
    if (xsm > 160 * 1024) {
        set_error("hessenberg: n=%d too large for the column buffer", n);
        return SC_BADINPUT;
    }
    SC_CUDA_TRY(cudaFuncSetAttribute(col_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024));
    const long long sA = (long long)n * n, sYV = (long long)n * NBH, sW = (long long)NBH * n;
    const double2 one = make_double2(1.0, 0.0), mone = make_double2(-1.0, 0.0), zero = make_double2(0.0, 0.0);
    for (int p = 0; p < npan; ++p) {
        const int k = p * NBH;
        const int ib = (n - 1 - k) < NBH ? (n - 1 - k) : NBH;
        int nch_prev = 0;
        for (int j = 0; j <= ib; ++j) {
            col_kernel<<<batch, CT, xsm, st>>>(P, n, k, j, ib, p, nch_prev);
            count_launch();
            if (j == ib) break;
            const int c0 = k + 1 + j;
            const int nch = (n - c0 + GCH - 1) / GCH;
            if (nch > 0) {
                dim3 g(nch, (n + GR - 1) / GR, batch);
                gemv_kernel<<<g, GR, 0, st>>>(P, n, c0, j);
                count_launch();
            }
            nch_prev = nch;
        }
        const int kc = k + ib;   // first trailing column
        if (kc < n) {
            const int nt = n - kc;
            // right: A[:, kc:] -= Y V[kc:, :]^H
            SC_TRY(zgemm_op(st, false, true, n, nt, ib, mone, P.Y, n, sYV, P.V + kc, n, sYV, one,
                            A + (long long)kc * n, n, sA, batch));
            // left: A[k+1:, kc:] -= V T^H V^H A[k+1:, kc:]
            const int mr = n - k - 1;
            SC_TRY(zgemm_op(st, true, false, ib, nt, mr, one, P.V + k + 1, n, sYV,
                            A + (long long)kc * n + k + 1, n, sA, zero, W, NBH, sW, batch));
            SC_TRY(zgemm_op(st, true, false, ib, nt, ib, one, P.T + (long long)p * NBH * NBH, NBH, P.sT, W, NBH,
                            sW, zero, W2, NBH, sW, batch));
            SC_TRY(zgemm_op(st, false, false, mr, nt, ib, mone, P.V + k + 1, n, sYV, W2, NBH, sW, one,
                            A + (long long)kc * n + k + 1, n, sA, batch));
        }
    }
    // ---- Q = P_0 P_1 ... accumulated from the last panel
    {
        dim3 g(gridfor(sA), batch);
        identity_clear_kernel<<<g, 256, 0, st>>>(Q, A, n);
        count_launch();
    }
    for (int p = npan - 1; p >= 0; --p) {
        const int k = p * NBH;
        const int ib = (n - 1 - k) < NBH ? (n - 1 - k) : NBH;
        const int mr = n - k - 1;
        dim3 g(gridfor((long long)n * ib), batch);
        panel_v_kernel<<<g, 256, 0, st>>>(A, n, k, ib, P.V);
        count_launch();
        double2* Qs = Q + (long long)(k + 1) * n + k + 1;
        SC_TRY(zgemm_op(st, true, false, ib, mr, mr, one, P.V + k + 1, n, sYV, Qs, n, sA, zero, W, NBH, sW, batch));
        SC_TRY(zgemm_op(st, false, false, ib, mr, ib, one, P.T + (long long)p * NBH * NBH, NBH, P.sT, W, NBH, sW,
                        zero, W2, NBH, sW, batch));
        SC_TRY(zgemm_op(st, false, false, mr, mr, ib, mone, P.V + k + 1, n, sYV, W2, NBH, sW, one, Qs, n, sA,
                        batch));
    }
    {
        dim3 g(gridfor(sA), batch);
        clear_below_kernel<<<g, 256, 0, st>>>(A, n);
        count_launch();
    }
    SC_CHECK_LAUNCH("hessenberg");
    return SC_OK;
}

}  // namespace sc
