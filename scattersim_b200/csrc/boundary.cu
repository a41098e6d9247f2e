// Boundary-system blocks of the scattervolume solve, batched over instances
// (ScatterVolume.cpp:339-466: MatTransfer, SetGaussianConstraints,
// SetBoundaryConditions).  Every kernel takes instance b = blockIdx.y; its
// order vectors live at svec + b * sv_stride as [Sx, Sy, Sz0, Sz1, EF (3 MF)]
// (column-major order index, MF each) and its wavenumber and top plane at
// kz0[2 b], kz0[2 b + 1].
#include "common.cuh"
#include "kernels.cuh"

namespace sc {

namespace {

// f3 dense (4MF x 3MF) (ScatterVolume.cpp:377-382)
__global__ void f3_kernel(int MF, const double2* __restrict__ svec, long long sv_stride, double2* __restrict__ F,
                          long long sF) {
    const int b = blockIdx.y;
    const double2* Sx = svec + b * sv_stride;
    const double2* Sy = Sx + MF;
    const double2* Sz1 = Sx + 3 * MF;
    double2* f = F + b * sF;
    const int n4 = 4 * MF;
    const long long tot = (long long)n4 * 3 * MF;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(t % n4), c = (int)(t / n4);
        const int rb = r / MF, ri = r % MF, cb = c / MF, ci = c % MF;
        double2 v = make_double2(0.0, 0.0);
        if (ri == ci) {
            if (rb == 0 && cb == 0) v = make_double2(-1.0, 0.0);
            else if (rb == 1 && cb == 1) v = make_double2(-1.0, 0.0);
            else if (rb == 2 && cb == 1) v = Sz1[ri];
            else if (rb == 2 && cb == 2) v = cneg(Sy[ri]);
            else if (rb == 3 && cb == 0) v = cneg(Sz1[ri]);
            else if (rb == 3 && cb == 2) v = Sx[ri];
        }
        f[t] = v;
    }
}

// The 6MF x 6MF boundary system except the Gd*inv(Gc)*f3 block, and b
// (ScatterVolume.cpp:398-414, 446, 456; f1/f2 of :357-373)
__global__ void system_kernel(int MF, const double2* __restrict__ svec, long long sv_stride,
                              const double* __restrict__ kz0, double2* __restrict__ Aall, long long sA,
                              double2* __restrict__ ball, long long sb) {
    const int inst = blockIdx.y;
    const double2* Sx = svec + inst * sv_stride;
    const double2* Sy = Sx + MF;
    const double2* Sz0 = Sx + 2 * MF;
    const double2* Sz1 = Sx + 3 * MF;
    const double2* EF = Sx + 4 * MF;
    const double k = kz0[2 * inst], z0 = kz0[2 * inst + 1];
    double2* A = Aall + inst * sA;
    double2* b = ball + inst * sb;
    const int n6 = 6 * MF;
    const long long tot = (long long)n6 * 3 * MF;   // columns 0..3MF
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(t % n6), c = (int)(t / n6);
        const int cb = c / MF, ci = c % MF;
        double2 v = make_double2(0.0, 0.0);
        if (r < MF) {
            // reflected Gauss row r: Sx R_x + Sy R_y - Sz0 R_z
            if (ci == r) v = (cb == 0) ? Sx[r] : (cb == 1) ? Sy[r] : cneg(Sz0[r]);
        } else if (r >= 2 * MF) {
            // f2 block at rows 2MF.., columns 0..3MF (transmitted Gauss rows
            // MF..2MF are zero here: they live in columns 3MF..6MF)
            const int rr = r - 2 * MF, rb = rr / MF, ri = rr % MF;
            if (ri == ci) {
                if (rb == 0 && cb == 0) v = make_double2(1.0, 0.0);
                else if (rb == 1 && cb == 1) v = make_double2(1.0, 0.0);
                else if (rb == 2 && cb == 1) v = Sz0[ri];
                else if (rb == 2 && cb == 2) v = Sy[ri];
                else if (rb == 3 && cb == 0) v = cneg(Sz0[ri]);
                else if (rb == 3 && cb == 2) v = cneg(Sx[ri]);
            }
        }
        A[(long long)c * n6 + r] = v;
    }
    // transmitted Gauss rows (MF..2MF) in columns 3MF..6MF, rows 0..2MF of those columns
    const long long tot2 = (long long)(2 * MF) * 3 * MF;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot2;
         t += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(t % (2 * MF)), c = 3 * MF + (int)(t / (2 * MF));
        const int cb = (c - 3 * MF) / MF, ci = (c - 3 * MF) % MF;
        double2 v = make_double2(0.0, 0.0);
        if (r >= MF && ci == r - MF) v = (cb == 0) ? Sx[ci] : (cb == 1) ? Sy[ci] : Sz1[ci];
        A[(long long)c * n6 + r] = v;
    }
    // b = [0 (2MF); -f1 EF]
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n6; r += gridDim.x * blockDim.x) {
        double2 v = make_double2(0.0, 0.0);
        if (r >= 2 * MF) {
            const int rr = r - 2 * MF, rb = rr / MF, ri = rr % MF;
            // phase = exp(i k z0 Sz0)
            const double2 ph = cexp(cscale(cmul(make_double2(0.0, k), Sz0[ri]), z0));
            const double2 ex = EF[ri], ey = EF[MF + ri], ez = EF[2 * MF + ri];
            double2 f;
            if (rb == 0) f = cmul(ph, ex);
            else if (rb == 1) f = cmul(ph, ey);
            else if (rb == 2) f = cadd(cneg(cmul(cmul(ph, Sz0[ri]), ey)), cmul(cmul(ph, Sy[ri]), ez));
            else f = csub(cmul(cmul(ph, Sz0[ri]), ex), cmul(cmul(ph, Sx[ri]), ez));
            v = cneg(f);
        }
        b[r] = v;
    }
}

// dst_b(rows x cols, ld ldd) = src_b(rows x cols, ld lds), per-batch pointers
__global__ void copy_block_kernel(int rows, int cols, const double2* const* __restrict__ src, int lds,
                                  double2* const* __restrict__ dst, int ldd) {
    const int b = blockIdx.y;
    const double2* s = src[b];
    double2* d = dst[b];
    const long long tot = (long long)rows * cols;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(t % rows), c = (int)(t / rows);
        d[(long long)c * ldd + r] = s[(long long)c * lds + r];
    }
}

// b rows 2MF.. of the boundary system: -f1 EF at row rb*MF + ri (ScatterVolume.cpp:456, f1 of :357-366)
__device__ __forceinline__ double2 rhs_row(int rb, int ri, int MF, const double2* Sx, const double2* Sy,
                                           const double2* Sz0, const double2* EF, double k, double z0) {
    const double2 ph = cexp(cscale(cmul(make_double2(0.0, k), Sz0[ri]), z0));
    const double2 ex = EF[ri], ey = EF[MF + ri], ez = EF[2 * MF + ri];
    double2 f;
    if (rb == 0) f = cmul(ph, ex);
    else if (rb == 1) f = cmul(ph, ey);
    else if (rb == 2) f = cadd(cneg(cmul(cmul(ph, Sz0[ri]), ey)), cmul(cmul(ph, Sy[ri]), ez));
    else f = csub(cmul(cmul(ph, Sz0[ri]), ex), cmul(cmul(ph, Sx[ri]), ez));
    return cneg(f);
}

// The 6MF system with R eliminated order by order (rows 0..2 of f2 and the
// reflected Gauss row give R_x, R_y, R_z of each order from T):
//   R_x = b0 - Y0 T,  R_y = b1 - Y1 T,  R_z = (Sx R_x + Sy R_y) / Sz0
// leaves, for T, the transmitted Gauss rows and rows 2 and 3 of f2:
//   K2 = Y2 - a2y Y1 - a2x Y0,  K3 = Y3 - a3x Y0 - a3y Y1  (per order m, Yi = rows i MF + m of Y)
//   a2y = Sz0 + Sy^2 / Sz0,  a2x = Sx Sy / Sz0,  a3x = -Sz0 - Sx^2 / Sz0,  a3y = -Sx Sy / Sz0
// Ared (3MF x 3MF) = [Gauss_T; K2; K3], bred = [0; b2 - a2y b1 - a2x b0; b3 - a3x b0 - a3y b1]
__global__ void reduced_kernel(int MF, const double2* __restrict__ svec, long long sv_stride,
                               const double* __restrict__ kz0, const double2* const* __restrict__ Yp, int ldy,
                               double2* __restrict__ Aall, long long sA, double2* __restrict__ ball, long long sb) {
    const int inst = blockIdx.y;
    const double2* Sx = svec + inst * sv_stride;
    const double2* Sy = Sx + MF;
    const double2* Sz0 = Sx + 2 * MF;
    const double2* Sz1 = Sx + 3 * MF;
    const double2* EF = Sx + 4 * MF;
    const double k = kz0[2 * inst], z0 = kz0[2 * inst + 1];
    const double2* Y = Yp[inst];
    double2* A = Aall + inst * sA;
    double2* b = ball + inst * sb;
    const int n3 = 3 * MF;
    const long long tot = (long long)n3 * n3;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(t % n3), c = (int)(t / n3);
        const int blk = r / MF, m = r % MF;
        double2 v;
        if (blk == 0) {
            const int cb = c / MF, ci = c % MF;
            v = (ci == m) ? ((cb == 0) ? Sx[m] : (cb == 1) ? Sy[m] : Sz1[m]) : make_double2(0.0, 0.0);
        } else {
            const double2 cx = cdiv(Sx[m], Sz0[m]), cy = cdiv(Sy[m], Sz0[m]);
            const double2* y = Y + (long long)c * ldy;
            const double2 y0 = y[m], y1 = y[MF + m];
            if (blk == 1) {
                const double2 a2y = cadd(Sz0[m], cmul(Sy[m], cy)), a2x = cmul(Sy[m], cx);
                v = csub(csub(y[2 * MF + m], cmul(a2y, y1)), cmul(a2x, y0));
            } else {
                const double2 a3x = cneg(cadd(Sz0[m], cmul(Sx[m], cx))), a3y = cneg(cmul(Sx[m], cy));
                v = csub(csub(y[3 * MF + m], cmul(a3x, y0)), cmul(a3y, y1));
            }
        }
        A[(long long)c * n3 + r] = v;
    }
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < MF; m += gridDim.x * blockDim.x) {
        const double2 cx = cdiv(Sx[m], Sz0[m]), cy = cdiv(Sy[m], Sz0[m]);
        const double2 b0 = rhs_row(0, m, MF, Sx, Sy, Sz0, EF, k, z0), b1 = rhs_row(1, m, MF, Sx, Sy, Sz0, EF, k, z0);
        const double2 b2 = rhs_row(2, m, MF, Sx, Sy, Sz0, EF, k, z0), b3 = rhs_row(3, m, MF, Sx, Sy, Sz0, EF, k, z0);
        const double2 a2y = cadd(Sz0[m], cmul(Sy[m], cy)), a2x = cmul(Sy[m], cx);
        const double2 a3x = cneg(cadd(Sz0[m], cmul(Sx[m], cx))), a3y = cneg(cmul(Sx[m], cy));
        b[m] = make_double2(0.0, 0.0);
        b[MF + m] = csub(csub(b2, cmul(a2y, b1)), cmul(a2x, b0));
        b[2 * MF + m] = csub(csub(b3, cmul(a3x, b0)), cmul(a3y, b1));
    }
}

// x = [R_x R_y R_z T] from T (the reduced solution) and Y
__global__ void recover_kernel(int MF, const double2* __restrict__ svec, long long sv_stride,
                               const double* __restrict__ kz0, const double2* const* __restrict__ Yp, int ldy,
                               const double2* __restrict__ Tall, long long sT, double2* const* __restrict__ xp) {
    const int inst = blockIdx.y;
    const double2* Sx = svec + inst * sv_stride;
    const double2* Sy = Sx + MF;
    const double2* Sz0 = Sx + 2 * MF;
    const double2* EF = Sx + 4 * MF;
    const double k = kz0[2 * inst], z0 = kz0[2 * inst + 1];
    const double2* Y = Yp[inst];
    const double2* T = Tall + inst * sT;
    double2* x = xp[inst];
    const int n3 = 3 * MF;
    for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < MF; m += gridDim.x * blockDim.x) {
        double2 s0 = make_double2(0.0, 0.0), s1 = make_double2(0.0, 0.0);
        for (int c = 0; c < n3; ++c) {
            const double2 tc = T[c];
            s0 = cfma(Y[(long long)c * ldy + m], tc, s0);
            s1 = cfma(Y[(long long)c * ldy + MF + m], tc, s1);
        }
        const double2 rx = csub(rhs_row(0, m, MF, Sx, Sy, Sz0, EF, k, z0), s0);
        const double2 ry = csub(rhs_row(1, m, MF, Sx, Sy, Sz0, EF, k, z0), s1);
        x[m] = rx;
        x[MF + m] = ry;
        x[2 * MF + m] = cadd(cmul(cdiv(Sx[m], Sz0[m]), rx), cmul(cdiv(Sy[m], Sz0[m]), ry));
    }
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n3; c += gridDim.x * blockDim.x) x[n3 + c] = T[c];
}

unsigned blocks_for(long long tot) {
    long long b = (tot + 255) / 256;
    if (b < 1) b = 1;
    if (b > 4096) b = 4096;
    return (unsigned)b;
}

}  // namespace

sc_status boundary_f3(cudaStream_t st, int MF, const double2* svec, long long sv_stride, double2* F, long long sF,
                      int count) {
    if (count <= 0) return SC_OK;
    f3_kernel<<<dim3(blocks_for(12LL * MF * MF), count), 256, 0, st>>>(MF, svec, sv_stride, F, sF);
    count_launch();
    SC_CHECK_LAUNCH("boundary_f3");
    return SC_OK;
}

sc_status boundary_system(cudaStream_t st, int MF, const double2* svec, long long sv_stride, const double* kz0,
                          double2* A6, long long sA, double2* b6, long long sb, int count) {
    if (count <= 0) return SC_OK;
    system_kernel<<<dim3(blocks_for(18LL * MF * MF), count), 256, 0, st>>>(MF, svec, sv_stride, kz0, A6, sA, b6,
                                                                           sb);
    count_launch();
    SC_CHECK_LAUNCH("boundary_system");
    return SC_OK;
}

sc_status boundary_reduced(cudaStream_t st, int MF, const double2* svec, long long sv_stride, const double* kz0,
                           const double2* const* Y, int ldy, double2* A3, long long sA, double2* b3, long long sb,
                           int count) {
    if (count <= 0) return SC_OK;
    reduced_kernel<<<dim3(blocks_for(9LL * MF * MF), count), 256, 0, st>>>(MF, svec, sv_stride, kz0, Y, ldy, A3, sA,
                                                                           b3, sb);
    count_launch();
    SC_CHECK_LAUNCH("boundary_reduced");
    return SC_OK;
}

sc_status boundary_recover(cudaStream_t st, int MF, const double2* svec, long long sv_stride, const double* kz0,
                           const double2* const* Y, int ldy, const double2* T, long long sT, double2* const* x,
                           int count) {
    if (count <= 0) return SC_OK;
    recover_kernel<<<dim3((3 * MF + 127) / 128, count), 128, 0, st>>>(MF, svec, sv_stride, kz0, Y, ldy, T, sT, x);
    count_launch();
    SC_CHECK_LAUNCH("boundary_recover");
    return SC_OK;
}

sc_status copy_blocks(cudaStream_t st, int rows, int cols, const double2* const* src, int lds, double2* const* dst,
                      int ldd, int count) {
    if (count <= 0 || rows <= 0 || cols <= 0) return SC_OK;
    copy_block_kernel<<<dim3(blocks_for((long long)rows * cols), count), 256, 0, st>>>(rows, cols, src, lds, dst,
                                                                                       ldd);
    count_launch();
    SC_CHECK_LAUNCH("copy_blocks");
    return SC_OK;
}

}  // namespace sc
