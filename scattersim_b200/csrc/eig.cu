// Batched non-Hermitian complex128 eigensolver: eigenvalues and right
// eigenvectors of `batch` n x n matrices, the job of LAPACKE_zgeev('N','V')
// behind MKL_eigensolve (third_Lapack.h:37-44, called at
// ScatterVolume.cpp:253-277).
//
// Pipeline (one CTA per matrix for the sequential phases):
//   1-2. hessenberg_blocked (hess.cu)  blocked Householder reduction to upper
//                     Hessenberg form and the explicit Q = H(0) ... H(n-2)
//                     (the initial Schur vectors).
//   3. hqr_kernel     complex single-shift QR to Schur form T = Z^H A Z with
//                     Ahues-Tisseur deflation.  Large active blocks take
//                     multishift sweeps: 16 shifts (eigenvalues of the trailing
//                     16 x 16 block) as a chain of single-shift bulges chased in
//                     lockstep by 16 warps through a 96 x 96 shared-memory
//                     window; the window's rotations are then streamed over the
//                     rows to the right, the columns above and the Schur vectors.
//                     Active blocks of <= 64 rows are finished in shared memory
//                     (Wilkinson shifts) with the accumulated unitary applied
//                     afterwards.
//   4. trevc_kernel   eigenvectors of T by back substitution, one warp per
//                     eigenvalue, small pivots raised to eps*|lambda|.
//   5. V = Z * Y      batched zgemm, then unit 2-norm columns (zgeev's
//                     normalisation; the largest component is made real).
// Every loop has an iteration cap; a matrix that hits it gets info > 0 and the
// kernel returns normally.
#include "common.cuh"
#include "kernels.cuh"

#include <cfloat>

#include <cooperative_groups.h>

namespace cg = cooperative_groups;

namespace sc {

namespace {
constexpr int HT = 512;     // threads per CTA of the QR kernel
constexpr int W = 64;       // shared-memory window
constexpr double ULP = DBL_EPSILON;
constexpr double SAFMIN = DBL_MIN;


// [c s; -conj(s) c] [f; g] = [r; 0], c real (no overflow scaling: the
// matrices here are O(1)-scaled; two FP64 rsqrt instead of hypot/divisions)
__device__ __forceinline__ void zlartg(double2 f, double2 g, double& c, double2& s) {
    const double f2 = cnorm2(f), g2 = cnorm2(g);
    if (g2 == 0.0) {
        c = 1.0;
        s = make_double2(0.0, 0.0);
        return;
    }
    if (f2 == 0.0) {
        const double rg = rsqrt(g2);
        c = 0.0;
        s = make_double2(g.x * rg, -g.y * rg);
        return;
    }
    const double rf = rsqrt(f2), rd = rsqrt(f2 + g2);
    c = f2 * rf * rd;
    s = cscale(cmulc(f, g), rf * rd);   // f conj(g) / (|f| d)
}
// rows: a' = c a + s b ; b' = c b - conj(s) a   (12 FP64 mul/fma)
__device__ __forceinline__ void rot_rows(double c, double2 s, double2& a, double2& b) {
    const double ax = fma(c, a.x, fma(s.x, b.x, -s.y * b.y));
    const double ay = fma(c, a.y, fma(s.x, b.y, s.y * b.x));
    const double bx = fma(c, b.x, -fma(s.x, a.x, s.y * a.y));
    const double by = fma(c, b.y, -fma(s.x, a.y, -s.y * a.x));
    a = make_double2(ax, ay);
    b = make_double2(bx, by);
}
// cols (right multiply by G^H): a' = a c + b conj(s) ; b' = b c - a s
__device__ __forceinline__ void rot_cols(double c, double2 s, double2& a, double2& b) {
    const double ax = fma(c, a.x, fma(b.x, s.x, b.y * s.y));
    const double ay = fma(c, a.y, fma(b.y, s.x, -b.x * s.y));
    const double bx = fma(c, b.x, -fma(a.x, s.x, -a.y * s.y));
    const double by = fma(c, b.y, -fma(a.x, s.y, a.y * s.x));
    a = make_double2(ax, ay);
    b = make_double2(bx, by);
}

// ------------------------------------------------------------------ hqr
constexpr int NSH = 16;   // shifts (bulges) per multishift sweep, one warp each
constexpr int WB = 96;    // chase window (rows/cols kept in shared memory)
constexpr int SEP = 3;    // rows between consecutive bulges of a chain
// odd leading dimensions: a warp's row operation reads one row across 32
// columns, conflict-free only when the column stride is not a multiple of 32 banks
constexpr int WL = W + 1;     // small block
constexpr int WBL = WB + 1;   // chase window

struct HqrSmem {
    union {
        struct {
            double2 Hs[W * WL];      // small block, column-major, ld WL
            double2 U[W * WL];       // its accumulated unitary
            double2 chunk[W * 33];   // staging for the small-block far products
        } s;
        double2 win[WB * WBL];       // chase window, column-major, ld WBL
    } u;
    double rc[WB][NSH];              // rotation q of bulge i in this window: [q][i]
    double2 rs[WB][NSH];
    int bpos[NSH], bstart[NSH], bcnt[NSH], boff[NSH];
    int pub[4];                      // published window: ws, we, steps, status (0 ready, 1 done, 2 fail)
    double2 shifts[NSH];
    int red_i[HT / 32];
    int s_int[8];
};

__device__ __forceinline__ double2& HS(HqrSmem& S, int i, int j) { return S.u.s.Hs[j * WL + i]; }
__device__ __forceinline__ double2& US(HqrSmem& S, int i, int j) { return S.u.s.U[j * WL + i]; }
__device__ __forceinline__ double2& WN(HqrSmem& S, int i, int j) { return S.u.win[j * WBL + i]; }

// Ahues-Tisseur deflation test for subdiagonal k (rows/cols relative to a
// column-major array with leading dimension ld); lo..hi is the active range.
__device__ bool negligible(const double2* H, long long ld, int k, int lo, int hi) {
    double2 hkk1 = H[(long long)(k - 1) * ld + k];
    double sub = cabs1(hkk1);
    if (sub <= SAFMIN * 1e3) return true;
    double2 a = H[(long long)(k - 1) * ld + k - 1], d = H[(long long)k * ld + k];
    double tst = cabs1(a) + cabs1(d);
    if (tst == 0.0) {
        if (k - 2 >= lo) tst += fabs(H[(long long)(k - 2) * ld + k - 1].x);
        if (k + 1 <= hi) tst += fabs(H[(long long)k * ld + k + 1].x);
    }
    if (sub <= ULP * tst) {
        double2 up = H[(long long)k * ld + k - 1];
        double ab = fmax(sub, cabs1(up)), ba = fmin(sub, cabs1(up));
        double2 dd = csub(a, d);
        double aa = fmax(cabs1(d), cabs1(dd)), bb = fmin(cabs1(d), cabs1(dd));
        double s = aa + ab;
        if (ba * (ab / s) <= fmax(SAFMIN * 1e3, ULP * (bb * (aa / s)))) return true;
    }
    return false;
}

// Wilkinson shift from the trailing 2x2 of the active block (zlahqr)
__device__ double2 wilkinson(double2 h11, double2 h12, double2 h21, double2 h22) {
    double2 t = h22;
    double2 u = cmul(csqrt(h12), csqrt(h21));
    double s = cabs1(u);
    if (s != 0.0) {
        double2 x = cscale(csub(h11, h22), 0.5);
        double sx = cabs1(x);
        s = fmax(s, sx);
        double2 xs = cscale(x, 1.0 / s), us = cscale(u, 1.0 / s);
        double2 y = cscale(csqrt(cadd(cmul(xs, xs), cmul(us, us))), s);
        if (sx > 0.0) {
            double2 xx = cscale(x, 1.0 / sx);
            if (xx.x * y.x + xx.y * y.y < 0.0) y = cneg(y);
        }
        t = csub(t, cmul(u, cdiv(u, cadd(x, y))));
    }
    return t;
}

// Single-shift QR of an m x m block held in S.Hs, run by one warp.  With
// ACC the rotations are accumulated into S.U (the block then lies in the full
// Schur form); without it only the eigenvalues (diagonal) matter.  Returns
// false on the iteration cap.
template <bool ACC>
__device__ bool small_qr_warp(HqrSmem& S, int m, int maxit) {
    const int lane = threadIdx.x & 31;
    int hi = m - 1;
    int its = 0, total = 0;
    while (hi >= 0) {
        int lo = hi;
        while (lo > 0 && !negligible(S.u.s.Hs, WL, lo, 0, hi)) --lo;
        if (lo > 0) {
            if (lane == 0) HS(S, lo, lo - 1) = make_double2(0.0, 0.0);
            __syncwarp();
        }
        if (lo == hi) {
            --hi;
            its = 0;
            continue;
        }
        if (++total > maxit) return false;
        ++its;
        double2 sh;
        if (its == 10) {
            sh = cadd(make_double2(0.75 * fabs(HS(S, lo + 1, lo).x), 0.0), HS(S, lo, lo));
        } else if (its == 20) {
            sh = cadd(make_double2(0.75 * fabs(HS(S, hi, hi - 1).x), 0.0), HS(S, hi, hi));
        } else {
            sh = wilkinson(HS(S, hi - 1, hi - 1), HS(S, hi - 1, hi), HS(S, hi, hi - 1), HS(S, hi, hi));
        }
        const int jend = ACC ? m : hi + 1;   // row ops extend to the block edge only when accumulating
        const int ibeg = ACC ? 0 : lo;
        for (int k = lo; k < hi; ++k) {
            double c;
            double2 s;
            if (k == lo)
                zlartg(csub(HS(S, lo, lo), sh), HS(S, lo + 1, lo), c, s);
            else
                zlartg(HS(S, k, k - 1), HS(S, k + 1, k - 1), c, s);
            const int c0 = (k == lo) ? lo : k - 1;
            for (int j = c0 + lane; j < jend; j += 32) {
                double2 a = HS(S, k, j), bb = HS(S, k + 1, j);
                rot_rows(c, s, a, bb);
                HS(S, k, j) = a;
                HS(S, k + 1, j) = bb;
            }
            __syncwarp();
            if (k > lo && lane == 0) HS(S, k + 1, k - 1) = make_double2(0.0, 0.0);
            const int r1 = (k + 2 < hi ? k + 2 : hi);
            for (int i = ibeg + lane; i <= r1; i += 32) {
                double2 a = HS(S, i, k), bb = HS(S, i, k + 1);
                rot_cols(c, s, a, bb);
                HS(S, i, k) = a;
                HS(S, i, k + 1) = bb;
            }
            if (ACC) {
                for (int i = lane; i < m; i += 32) {
                    double2 a = US(S, i, k), bb = US(S, i, k + 1);
                    rot_cols(c, s, a, bb);
                    US(S, i, k) = a;
                    US(S, i, k + 1) = bb;
                }
            }
            __syncwarp();
        }
    }
    return true;
}

// Far updates after a small block [lo, lo+m) finished with unitary U.
__device__ void small_block_far(HqrSmem& S, double2* H, double2* Z, int n, int lo, int m) {
    const int tid = threadIdx.x;
    const int hi1 = lo + m;  // exclusive
    // right: H[lo:hi1, hi1:n] <- U^H * H[lo:hi1, hi1:n]
    for (int j0 = hi1; j0 < n; j0 += 32) {
        const int nc = (n - j0) < 32 ? (n - j0) : 32;
        for (int t = tid; t < m * nc; t += HT) {
            int r = t % m, c = t / m;
            S.u.s.chunk[c * WL + r] = H[(long long)(j0 + c) * n + lo + r];
        }
        __syncthreads();
        for (int t = tid; t < m * nc; t += HT) {
            int r = t % m, c = t / m;
            double2 acc = make_double2(0.0, 0.0);
            for (int l = 0; l < m; ++l) acc = cfma(cconj(US(S, l, r)), S.u.s.chunk[c * WL + l], acc);
            H[(long long)(j0 + c) * n + lo + r] = acc;
        }
        __syncthreads();
    }
    // above: H[0:lo, lo:hi1] <- H[0:lo, lo:hi1] * U ; Z[0:n, lo:hi1] <- Z * U
    for (int pass = 0; pass < 2; ++pass) {
        double2* X = pass == 0 ? H : Z;
        const int rows = pass == 0 ? lo : n;
        for (int i0 = 0; i0 < rows; i0 += 32) {
            const int nr = (rows - i0) < 32 ? (rows - i0) : 32;
            for (int t = tid; t < m * nr; t += HT) {
                int r = t % nr, c = t / nr;
                S.u.s.chunk[c * 33 + r] = X[(long long)(lo + c) * n + i0 + r];
            }
            __syncthreads();
            for (int t = tid; t < m * nr; t += HT) {
                int r = t % nr, c = t / nr;
                double2 acc = make_double2(0.0, 0.0);
                for (int l = 0; l < m; ++l) acc = cfma(S.u.s.chunk[l * 33 + r], US(S, l, c), acc);
                X[(long long)(lo + c) * n + i0 + r] = acc;
            }
            __syncthreads();
        }
    }
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::); }

// Applies a window's recorded rotations outside the window, in their true
// step order: tiles of 64 far columns (row rotations, rows [ws, we)) and of
// 64 far rows (column rotations, columns [ws, we)) are staged in shared
// memory with cp.async; each tile vector is owned by 16 lanes, lane i applying
// bulge i's rotation of the current step (same-step rotations touch disjoint
// rows).  A lane keeps the row its bulge carries forward in a register, so a
// rotation costs one shared-memory load and one store; each lane serves two
// vectors for instruction-level parallelism.
__device__ void far_apply(HqrSmem& S, double2* H, double2* Z, int n, int ws, int we, int ns, int steps,
                          long long* cyc, int crank, int csize) {
    const long long tf0 = clock64();
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const int wm = we - ws;
    constexpr int TV = 64;                    // vectors per tile
    const int bi = lane & 15;                 // bulge of this lane
    const int va = 2 * wid + (lane >> 4);     // first vector (0..31); second is va + 32
    const int vb = va + 32;
    const bool lane_ok = bi < ns;
    const int bst = lane_ok ? S.bstart[bi] - ws : 0;
    const int bof = lane_ok ? S.boff[bi] : 0;
    const int bct = lane_ok ? S.bcnt[bi] : 0;
    double2* stage = S.u.win;
    constexpr int LDC = WB + 1;               // column tile leading dimension (elements per vector)
    constexpr int LDR = TV + 1;               // row tile leading dimension (vectors per column)
    static_assert(TV * LDC <= WB * WBL && WB * LDR <= WB * WBL, "tile exceeds the window buffer");
    // rows [ws, we) of columns [we, n): row rotations
    for (int j0 = we + crank * TV; j0 < n; j0 += TV * csize) {
        const int nc = (n - j0) < TV ? (n - j0) : TV;
        for (int q = tid; q < wm * nc; q += HT) {
            const int r = q % wm, c = q / wm;
            cp_async16(&stage[c * LDC + r], &H[(long long)(j0 + c) * n + ws + r]);
        }
        cp_async_wait_all();
        __syncthreads();
        const bool oa = lane_ok && va < nc, ob = lane_ok && vb < nc;
        double2* pa = stage + va * LDC;
        double2* pb = stage + vb * LDC;
        double2 ca = make_double2(0.0, 0.0), cb = make_double2(0.0, 0.0);
        for (int tau = 0; tau < steps; ++tau) {
            const int q = tau - bof;
            if (q >= 0 && q < bct) {
                const int r = bst + q;
                const double c = S.rc[q][bi];
                const double2 sn = S.rs[q][bi];
                if (oa) {
                    if (q == 0) ca = pa[r];
                    double2 nx = pa[r + 1];
                    rot_rows(c, sn, ca, nx);
                    pa[r] = ca;
                    ca = nx;
                    if (q == bct - 1) pa[r + 1] = ca;
                }
                if (ob) {
                    if (q == 0) cb = pb[r];
                    double2 nx = pb[r + 1];
                    rot_rows(c, sn, cb, nx);
                    pb[r] = cb;
                    cb = nx;
                    if (q == bct - 1) pb[r + 1] = cb;
                }
            }
            __syncwarp();
        }
        __syncthreads();
        for (int q = tid; q < wm * nc; q += HT) {
            const int r = q % wm, c = q / wm;
            H[(long long)(j0 + c) * n + ws + r] = stage[c * LDC + r];
        }
        __syncthreads();
    }
    const long long tf1 = clock64();
    if (threadIdx.x == 0) cyc[3] += tf1 - tf0;
    // rows [0, ws) of H and [0, n) of Z, columns [ws, we): column rotations
    const int rows_total = ws + n;
    for (int i0 = crank * TV; i0 < rows_total; i0 += TV * csize) {
        const int nr = (rows_total - i0) < TV ? (rows_total - i0) : TV;
        for (int q = tid; q < wm * nr; q += HT) {
            const int rr = q % nr, c = q / nr;
            const int g = i0 + rr;
            const double2* src = (g < ws) ? (H + g) : (Z + (g - ws));
            cp_async16(&stage[c * LDR + rr], &src[(long long)(ws + c) * n]);
        }
        cp_async_wait_all();
        __syncthreads();
        const bool oa = lane_ok && va < nr, ob = lane_ok && vb < nr;
        double2 ca = make_double2(0.0, 0.0), cb = make_double2(0.0, 0.0);
        for (int tau = 0; tau < steps; ++tau) {
            const int q = tau - bof;
            if (q >= 0 && q < bct) {
                const int cc = bst + q;
                const double c = S.rc[q][bi];
                const double2 sn = S.rs[q][bi];
                if (oa) {
                    if (q == 0) ca = stage[cc * LDR + va];
                    double2 nx = stage[(cc + 1) * LDR + va];
                    rot_cols(c, sn, ca, nx);
                    stage[cc * LDR + va] = ca;
                    ca = nx;
                    if (q == bct - 1) stage[(cc + 1) * LDR + va] = ca;
                }
                if (ob) {
                    if (q == 0) cb = stage[cc * LDR + vb];
                    double2 nx = stage[(cc + 1) * LDR + vb];
                    rot_cols(c, sn, cb, nx);
                    stage[cc * LDR + vb] = cb;
                    cb = nx;
                    if (q == bct - 1) stage[(cc + 1) * LDR + vb] = cb;
                }
            }
            __syncwarp();
        }
        __syncthreads();
        for (int q = tid; q < wm * nr; q += HT) {
            const int rr = q % nr, c = q / nr;
            const int g = i0 + rr;
            double2* dst = (g < ws) ? (H + g) : (Z + (g - ws));
            dst[(long long)(ws + c) * n] = stage[c * LDR + rr];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) cyc[4] += clock64() - tf1;
}

// One multishift sweep over the active block [lo, ihi] with ns shifts in
// S.shifts.  The ns single-shift bulges are introduced SEP rows apart and
// advanced in lockstep: every step, warp i computes bulge i's rotation and
// applies it to its two rows (phase 1), then to its two columns (phase 2).
// Rotations of different bulges act on disjoint rows / disjoint columns and
// row and column operations commute, so each phase runs in parallel.  The
// chase stays inside a WB x WB shared-memory window; at the end of a window
// the recorded rotations are applied to the rows to its right, the columns
// above it and the Schur vectors.  There they are applied bulge by bulge
// (front bulge first): two rotations of different bulges that touch a common
// row are, in the true step order, already front-bulge first, and all other
// pairs commute, so the reordering is exact.
__device__ bool multishift_sweep(HqrSmem& S, double2* H, double2* Z, int n, int lo, int ihi, int ns,
                                 long long* cyc, int crank, int csize) {
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    cg::cluster_group cluster = cg::this_cluster();
    if (crank == 0 && tid < NSH) {
        S.bpos[tid] = lo;
        S.bcnt[tid] = 0;
    }
    __syncthreads();
    int t = 0;   // global step (bulge i is introduced at step SEP*i)
    while (true) {
        if (crank == 0) {
            // ---- rank 0: next window and the chase through it
            int front = -1, rear = -1;
            for (int i = 0; i < ns; ++i) {
                bool done = S.bpos[i] > ihi - 1;
                bool intro = t >= SEP * i || S.bpos[i] > lo;
                if (!done && front < 0) front = i;
                if (!done && intro) rear = i;
            }
            if (front < 0) {
                if (tid == 0) S.pub[3] = 1;
            } else {
                const bool all_intro = (SEP * (ns - 1) <= t) || S.bpos[ns - 1] > lo;
                const int ws = all_intro ? (S.bpos[rear] - 1 > lo ? S.bpos[rear] - 1 : lo) : lo;
                const int we = (ws + WB < ihi + 1) ? ws + WB : ihi + 1;
                const int wm = we - ws;
                for (int q = tid; q < WB * WB; q += HT) {
                    int i = q % WB, j = q / WB;
                    WN(S, i, j) = (i < wm && j < wm) ? H[(long long)(ws + j) * n + ws + i] : make_double2(0.0, 0.0);
                }
                if (tid < NSH) {
                    S.bstart[tid] = S.bpos[tid];
                    S.bcnt[tid] = 0;
                    S.boff[tid] = 0;
                }
                __syncthreads();
                const long long tch = clock64();
                int steps = 0;
                while (true) {
                    // front bulge of this step and its room in the window
                    int fr = -1;
                    for (int i = 0; i < ns; ++i)
                        if (S.bpos[i] <= ihi - 1) {
                            fr = i;
                            break;
                        }
                    if (fr < 0) break;
                    const int rf = S.bpos[fr];
                    if (!(rf + 2 <= we - 1 || we == ihi + 1)) break;
                    // phase 1: rotations and row operations
                    double c = 1.0;
                    double2 sn = make_double2(0.0, 0.0);
                    int r = -1;
                    bool act = false, intro = false;
                    if (wid < ns) {
                        r = S.bpos[wid];
                        intro = (t == SEP * wid);
                        act = (r <= ihi - 1) && (intro || r > lo);
                        if (act) {
                            const int lr = r - ws;
                            if (intro)
                                zlartg(csub(WN(S, lr, lr), S.shifts[wid]), WN(S, lr + 1, lr), c, sn);
                            else
                                zlartg(WN(S, lr, lr - 1), WN(S, lr + 1, lr - 1), c, sn);
                            const int c0 = intro ? lr : lr - 1;
                            for (int j = c0 + lane; j < wm; j += 32) {
                                double2 a = WN(S, lr, j), bb = WN(S, lr + 1, j);
                                rot_rows(c, sn, a, bb);
                                WN(S, lr, j) = a;
                                WN(S, lr + 1, j) = bb;
                            }
                            __syncwarp();
                            if (lane == 0) {
                                if (!intro) WN(S, lr + 1, lr - 1) = make_double2(0.0, 0.0);
                                if (S.bcnt[wid] == 0) S.boff[wid] = steps;
                                S.rc[S.bcnt[wid]][wid] = c;
                                S.rs[S.bcnt[wid]][wid] = sn;
                            }
                        }
                    }
                    __syncthreads();
                    // phase 2: column operations
                    if (act) {
                        const int lr = r - ws;
                        const int r1 = ((r + 2 < ihi) ? r + 2 : ihi) - ws;
                        for (int i = lane; i <= r1; i += 32) {
                            double2 a = WN(S, i, lr), bb = WN(S, i, lr + 1);
                            rot_cols(c, sn, a, bb);
                            WN(S, i, lr) = a;
                            WN(S, i, lr + 1) = bb;
                        }
                        if (lane == 0) {
                            S.bcnt[wid] += 1;
                            S.bpos[wid] = r + 1;
                        }
                    }
                    ++t;
                    ++steps;
                    __syncthreads();
                }
                if (tid == 0) cyc[2] += clock64() - tch;
                for (int q = tid; q < wm * wm; q += HT) {
                    int i = q % wm, j = q / wm;
                    H[(long long)(ws + j) * n + ws + i] = WN(S, i, j);
                }
                if (tid == 0) {
                    S.pub[0] = ws;
                    S.pub[1] = we;
                    S.pub[2] = steps;
                    // no room to move cannot happen with WB >= SEP*NSH + 8; fail instead of spinning
                    S.pub[3] = steps == 0 ? 2 : 0;
                }
            }
        }
        // ---- publish the window to the cluster
        cluster.sync();
        if (crank != 0) {
            HqrSmem* S0 = cluster.map_shared_rank(&S, 0);
            if (tid < 4) S.pub[tid] = S0->pub[tid];
            if (tid < NSH) {
                S.bstart[tid] = S0->bstart[tid];
                S.boff[tid] = S0->boff[tid];
                S.bcnt[tid] = S0->bcnt[tid];
            }
            // rotations recorded per bulge: at most WB - 1 (a bulge crosses the window
            // once), even when window steps exceed WB while bulges are introduced
            int qmax = 0;
            for (int i = 0; i < NSH; ++i) qmax = max(qmax, S0->bcnt[i]);
            qmax = min(qmax, WB);
            for (int q = tid; q < qmax * NSH; q += HT) {
                const int qq = q / NSH, i = q % NSH;
                S.rc[qq][i] = S0->rc[qq][i];
                S.rs[qq][i] = S0->rs[qq][i];
            }
        }
        __syncthreads();
        const int status = S.pub[3];
        if (status != 0) {
            // every rank has read rank 0's shared memory before any rank leaves
            cluster.sync();
            return status == 1;
        }
        far_apply(S, H, Z, n, S.pub[0], S.pub[1], ns, S.pub[2], cyc, crank, csize);
        cluster.sync();
    }
}

__global__ void __launch_bounds__(HT, 1)
hqr_kernel(double2* Hall, double2* Zall, int n, long long sA, double2* wall, int* info,
           int maxsweeps, long long* stats) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    HqrSmem& S = *reinterpret_cast<HqrSmem*>(smem_raw);
    cg::cluster_group cluster = cg::this_cluster();
    const int crank = (int)cluster.block_rank(), csize = (int)cluster.num_blocks();
    const int b = blockIdx.x / csize, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    double2* H = Hall + b * sA;
    double2* Z = Zall + b * sA;
    double2* w = wall + (long long)b * n;
    int ihi = n - 1, its = 0, sweeps = 0;
    bool failed = false;
    // phase cycle counters (thread 0): shifts, chase, far-right, far-rows, small blocks
    long long cyc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    long long t0 = clock64();
    // Every rank of the cluster evaluates the control decisions (deflation
    // point, shifts) from the same global data with the same code, so all
    // ranks take the same branches and the same cluster barriers.  The
    // negligible subdiagonal is left in place (no rotation ever touches it
    // again), so no rank's decision depends on another rank's write.
    while (ihi >= 0) {
        // ---- deflation point: largest k in (0, ihi] with negligible H[k, k-1]
        int best = 0;
        for (int k = ihi - tid; k >= 1; k -= HT) {
            if (negligible(H, n, k, 0, ihi)) {
                best = k;
                break;
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) best = max(best, __shfl_xor_sync(0xffffffffu, best, o));
        if (lane == 0) S.red_i[wid] = best;
        __syncthreads();
        if (tid == 0) {
            int bb = 0;
            for (int q = 0; q < HT / 32; ++q) bb = max(bb, S.red_i[q]);
            S.s_int[0] = bb;
        }
        __syncthreads();
        const int lo = S.s_int[0];
        __syncthreads();
        if (lo == ihi) {
            if (crank == 0 && tid == 0) w[ihi] = H[(long long)ihi * n + ihi];
            --ihi;
            its = 0;
            continue;
        }
        const int m = ihi - lo + 1;
        if (m <= W) {
            // ---- rank 0 finishes the block in shared memory
            const long long tsm = clock64();
            if (crank == 0) {
                for (int q = tid; q < W * W; q += HT) {
                    int i = q % W, j = q / W;
                    HS(S, i, j) = (i < m && j < m) ? H[(long long)(lo + j) * n + lo + i] : make_double2(0.0, 0.0);
                    US(S, i, j) = make_double2(i == j ? 1.0 : 0.0, 0.0);
                }
                __syncthreads();
                if (wid == 0) {
                    bool ok = small_qr_warp<true>(S, m, 30 * m + 30);
                    if (lane == 0) S.s_int[1] = ok ? 1 : 0;
                }
                __syncthreads();
                for (int q = tid; q < m * m; q += HT) {
                    int i = q % m, j = q / m;
                    H[(long long)(lo + j) * n + lo + i] = HS(S, i, j);
                }
                __syncthreads();
                small_block_far(S, H, Z, n, lo, m);
                for (int k = lo + tid; k <= ihi; k += HT) w[k] = HS(S, k - lo, k - lo);
            }
            cluster.sync();
            const int ok = (crank == 0) ? S.s_int[1] : cluster.map_shared_rank(&S, 0)->s_int[1];
            cluster.sync();
            if (tid == 0) cyc[5] += clock64() - tsm;
            if (!ok) {
                failed = true;
                break;
            }
            ihi = lo - 1;
            its = 0;
            continue;
        }
        if (++sweeps > maxsweeps) {
            failed = true;
            break;
        }
        ++its;
        // ---- shifts: eigenvalues of the trailing ns x ns block (every rank)
        const long long tsh = clock64();
        const int ns = NSH;
        for (int q = tid; q < W * W; q += HT) {
            int i = q % W, j = q / W;
            HS(S, i, j) = (i < ns && j < ns) ? H[(long long)(ihi - ns + 1 + j) * n + ihi - ns + 1 + i]
                                             : make_double2(0.0, 0.0);
        }
        __syncthreads();
        if (wid == 0) small_qr_warp<false>(S, ns, 30 * ns);
        __syncthreads();
        if (tid < ns) {
            double2 sh = HS(S, tid, tid);
            if (its % 6 == 0) {
                // exceptional shifts: perturb by the size of the last subdiagonal
                double e = 0.75 * cabs1(H[(long long)(ihi - 1) * n + ihi]);
                sh = cadd(sh, make_double2(e * (1.0 + 0.1 * tid), 0.0));
            }
            S.shifts[tid] = sh;
        }
        __syncthreads();
        if (tid == 0) cyc[1] += clock64() - tsh;
        if (!multishift_sweep(S, H, Z, n, lo, ihi, ns, cyc, crank, csize)) {
            failed = true;
            break;
        }
    }
    if (crank == 0 && tid == 0 && info != nullptr) info[b] = failed ? (ihi + 1 > 0 ? ihi + 1 : 1) : 0;
    if (crank == 0 && tid == 0 && stats != nullptr) {
        cyc[7] = clock64() - t0;
        stats[(long long)b * 8 + 0] = sweeps;
        for (int q = 1; q < 8; ++q) stats[(long long)b * 8 + q] = cyc[q];
    }
    cluster.sync();   // no rank leaves while another may still read its shared memory
}

// ------------------------------------------------------------------ trevc
// Y[:, k] = eigenvector of upper triangular T for T[k,k] (Y upper triangular).
__global__ void trevc_kernel(const double2* Tall, double2* Yall, int n, long long sA) {
    const int b = blockIdx.y;
    const int warps = blockDim.x >> 5;
    const int k = blockIdx.x * warps + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (k >= n) return;
    const double2* T = Tall + b * sA;
    double2* y = Yall + b * sA + (long long)k * n;
    const double2 lam = T[(long long)k * n + k];
    const double smin = fmax(ULP * cabs1(lam), SAFMIN * 1e3);
    for (int i = lane; i < n; i += 32) {
        if (i < k) y[i] = cneg(T[(long long)k * n + i]);
        else y[i] = make_double2(i == k ? 1.0 : 0.0, 0.0);
    }
    __syncwarp();
    for (int j = k - 1; j >= 0; --j) {
        double2 d = csub(T[(long long)j * n + j], lam);
        if (cabs1(d) < smin) d = make_double2(smin, 0.0);
        double2 xj = cdiv(y[j], d);
        __syncwarp();
        if (lane == 0) y[j] = xj;
        const double2* tc = T + (long long)j * n;
        for (int i = lane; i < j; i += 32) y[i] = csub(y[i], cmul(tc[i], xj));
        __syncwarp();
    }
}

// unit 2-norm columns, largest-magnitude component made real and positive
__global__ void normalize_cols_kernel(double2* Vall, int rows, int cols, int ld, long long sA) {
    const int b = blockIdx.y;
    const int warps = blockDim.x >> 5;
    const int c = blockIdx.x * warps + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (c >= cols) return;
    double2* v = Vall + b * sA + (long long)c * ld;
    double s = 0.0, best = -1.0;
    int bi = 0;
    for (int i = lane; i < rows; i += 32) {
        double q = cnorm2(v[i]);
        s += q;
        if (q > best) { best = q; bi = i; }
    }
    s = warp_sum(s);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double ob = __shfl_xor_sync(0xffffffffu, best, o);
        int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
    }
    if (s == 0.0) return;
    double2 big = v[bi];
    double bm = cabs(big);
    double inv = 1.0 / sqrt(s);
    double2 ph = (bm > 0.0) ? make_double2(big.x / bm * inv, -big.y / bm * inv) : make_double2(inv, 0.0);
    __syncwarp();
    for (int i = lane; i < rows; i += 32) v[i] = cmul(v[i], ph);
}

}  // namespace

size_t hqr_smem_bytes() { return sizeof(HqrSmem); }

sc_status eig_batched(cudaStream_t st, double2* A, int n, int batch, double2* evl, double2* V,
                      int* info, Workspace& ws) {
    if (n <= 0 || batch <= 0) return SC_OK;
    if (batch > 65535) {
        set_error("eig: batch %d too large", batch);
        return SC_BADINPUT;
    }
    const long long sA = (long long)n * n;
    double2* Z = nullptr;
    SC_TRY(ws.get(&Z, (size_t)batch * sA, WS_EIG_Z, st));
    // per-device attributes; cheap host calls, set on every use so that any
    // device current on this thread is covered
    SC_CUDA_TRY(cudaFuncSetAttribute(hqr_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)sizeof(HqrSmem)));
    SC_TRY(hessenberg_blocked(st, A, n, batch, Z, ws));
    for (auto& e : ws.ev_hqr)
        if (!e) SC_CUDA_TRY(cudaEventCreate(&e));
    SC_TRY(ws.get(&ws.hqr_stats, (size_t)batch * 8, WS_STATS, st));
    ws.hqr_batch = batch;
    SC_CUDA_TRY(cudaEventRecord(ws.ev_hqr[0], st));
    {
        // clusters of up to 4 CTAs per matrix when the batch leaves SMs idle
        int dev = 0, sms = 148;
        SC_CUDA_TRY(cudaGetDevice(&dev));
        SC_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        int cl = 1;
        while (cl < 4 && (long long)batch * cl * 2 <= sms && n > 2 * W) cl *= 2;
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3((unsigned)(batch * cl));
        cfg.blockDim = dim3(HT);
        cfg.dynamicSmemBytes = sizeof(HqrSmem);
        cfg.stream = st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = cl;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        SC_CUDA_TRY(cudaLaunchKernelEx(&cfg, hqr_kernel, A, Z, n, sA, evl, info, 60 * n + 100, ws.hqr_stats));
        count_launch();
    }
    SC_CUDA_TRY(cudaEventRecord(ws.ev_hqr[1], st));
    SC_CHECK_LAUNCH("hqr");
    // Y (upper triangular eigenvectors of T) into V, then V = Z * Y
    double2* Y = nullptr;
    SC_TRY(ws.get(&Y, (size_t)batch * sA, WS_EIG_Y, st));
    {
        const int warps = 8;
        dim3 g((n + warps - 1) / warps, batch);
        trevc_kernel<<<g, 32 * warps, 0, st>>>(A, Y, n, sA);
        count_launch();
    }
    SC_TRY(zgemm(st, n, n, n, make_double2(1.0, 0.0), Z, n, sA, Y, n, sA, make_double2(0.0, 0.0), V, n,
                 sA, batch));
    {
        const int warps = 8;
        dim3 g((n + warps - 1) / warps, batch);
        normalize_cols_kernel<<<g, 32 * warps, 0, st>>>(V, n, n, n, sA);
        count_launch();
    }
    SC_CHECK_LAUNCH("eig");
    return SC_OK;
}

sc_status normalize_columns(cudaStream_t st, double2* V, int rows, int cols, int ld, long long sA,
                            int batch) {
    const int warps = 8;
    dim3 g((cols + warps - 1) / warps, batch);
    normalize_cols_kernel<<<g, 32 * warps, 0, st>>>(V, rows, cols, ld, sA);
    count_launch();
    SC_CHECK_LAUNCH("normalize");
    return SC_OK;
}

}  // namespace sc
