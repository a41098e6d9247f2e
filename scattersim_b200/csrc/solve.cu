// The scattervolume solve on the device (ScatterVolume.cpp:573-902).
//
// Stage map (reference -> here):
//   volume::CalculateD, phi         fft2_crop + assemble_bc (Phi = [[0,B],[C,0]])
//   EigenDecompositionD / zgeev     eig of Omega = B C (2M x 2M), then the 4M
//                                   eigenpairs of Phi: lambda = +-sqrt(mu),
//                                   vector [w; C w / lambda]
//   Eigen_Sort pairing              even slot = root with Im > 0 (Re > 0 if
//                                   real): the forward mode; odd = its negative
//   Gd/Gc + Gc_static chain         GD_i = V diag(1|Di), GC_i = V diag(Ci|1);
//                                   Gc_static <- GC_i GD_i^-1 Gc_static via
//                                   LU(GD_i) and a solve with Gc_static
//   SetBoundaryConditions + zgesv   A[2M:, 3M:] = GD_0 Gc_static^-1 f3, LU solve
//   Beta chain, Q, Pz               LU solves with the stored GD_i factors,
//                                   column scaling, Pz as a batched product
// Eigenvalue pairing and eigenvector scale differ from the reference's MKL
// output; every quantity passed out (x, fields of Qc/Qh at each boundary)
// is invariant to both.
#include "context.cuh"

#include <cmath>
#include <cstring>

namespace sc {

namespace {

// ------------------------------------------------------------------ kernels

// V (n4 x n4) and evl (n4) of one layer from mu (n2), W (n2 x n2), CW = C W
__global__ void build_v_kernel(const double2* __restrict__ mu, const double2* __restrict__ Wm,
                               const double2* __restrict__ CW, int n2, double2* __restrict__ V,
                               double2* __restrict__ evl) {
    const int z = blockIdx.y;
    const int n4 = 2 * n2;
    const long long tot = (long long)n4 * n4;
    const double2* m = mu + (long long)z * n2;
    const double2* w = Wm + (long long)z * n2 * n2;
    const double2* cw = CW + (long long)z * n2 * n2;
    double2* v = V + (long long)z * tot;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(t % n4), c = (int)(t / n4);
        const int j = c >> 1;
        double2 lam = csqrt(m[j]);
        if (lam.y < 0.0 || (lam.y == 0.0 && lam.x < 0.0)) lam = cneg(lam);
        if (cabs1(lam) == 0.0) lam = make_double2(1e-300, 0.0);
        const bool odd = (c & 1);
        double2 val;
        if (r < n2) {
            val = w[(long long)j * n2 + r];
        } else {
            val = cdiv(cw[(long long)j * n2 + (r - n2)], lam);
            if (odd) val = cneg(val);
        }
        v[t] = val;
        if (r == 0) evl[(long long)z * n4 + c] = odd ? cneg(lam) : lam;
    }
}

// per-layer column scales: dG = (1 even, Di odd), cG = (Ci even, 1 odd)
// (ScatterVolume.cpp:297-321)
__global__ void gdgc_scale_kernel(const double2* __restrict__ evl, int n4, int Z, const double* __restrict__ zpl,
                                  double k, double2* __restrict__ dG, double2* __restrict__ cG) {
    const int z = blockIdx.y;
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n4) return;
    double dzc, dzd;
    if (Z == 1) {
        dzc = zpl[Z] - zpl[0];
        dzd = zpl[0] - zpl[Z];
    } else {
        dzc = zpl[z + 1] - zpl[z];
        dzd = zpl[z] - zpl[z + 1];
    }
    const double2 lam = evl[(long long)z * n4 + j];
    // i * k * lambda * dz
    const double2 ik = make_double2(0.0, k);
    const double2 ac = cscale(cmul(ik, lam), dzc);
    const double2 ad = cscale(cmul(ik, lam), dzd);
    double2 d, c;
    if (j & 1) {
        d = cexp(ad);
        c = make_double2(1.0, 0.0);
    } else {
        d = make_double2(1.0, 0.0);
        c = cexp(ac);
    }
    dG[(long long)z * n4 + j] = d;
    cG[(long long)z * n4 + j] = c;
}

// out = in * diag(s) (column scaling), batched with strides
__global__ void scale_cols_kernel(const double2* __restrict__ in, long long sIn, const double2* __restrict__ s,
                                  long long sS, int rows, int cols, double2* __restrict__ out, long long sOut) {
    const int z = blockIdx.y;
    const long long tot = (long long)rows * cols;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x) {
        const int c = (int)(t / rows);
        out[z * sOut + t] = cmul(in[z * sIn + t], s[z * sS + c]);
    }
}

// out_z = diag(s_z) in_z (row scaling), batched
__global__ void scale_rows_batched_kernel(const double2* __restrict__ in, long long sIn,
                                          const double2* __restrict__ s, long long sS, int rows, int cols,
                                          double2* __restrict__ out, long long sOut) {
    const int z = blockIdx.y;
    const long long tot = (long long)rows * cols;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(t % rows);
        out[z * sOut + t] = cmul(in[z * sIn + t], s[z * sS + r]);
    }
}

// rhs0 = f1 EF + f2 R  (ScatterVolume.cpp:768-772)
__global__ void beta0_rhs_kernel(int MF, const double2* __restrict__ Sx, const double2* __restrict__ Sy,
                                 const double2* __restrict__ Sz0, const double2* __restrict__ EF,
                                 const double2* __restrict__ x, double k, double z0, double2* __restrict__ out) {
    const int n4 = 4 * MF;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < n4; r += gridDim.x * blockDim.x) {
        const int rb = r / MF, ri = r % MF;
        const double2 ph = cexp(cscale(cmul(make_double2(0.0, k), Sz0[ri]), z0));
        const double2 ex = EF[ri], ey = EF[MF + ri], ez = EF[2 * MF + ri];
        const double2 rx = x[ri], ry = x[MF + ri], rz = x[2 * MF + ri];
        double2 f1, f2;
        if (rb == 0) {
            f1 = cmul(ph, ex);
            f2 = rx;
        } else if (rb == 1) {
            f1 = cmul(ph, ey);
            f2 = ry;
        } else if (rb == 2) {
            f1 = cadd(cneg(cmul(cmul(ph, Sz0[ri]), ey)), cmul(cmul(ph, Sy[ri]), ez));
            f2 = cadd(cmul(Sz0[ri], ry), cmul(Sy[ri], rz));
        } else {
            f1 = csub(cmul(cmul(ph, Sz0[ri]), ex), cmul(cmul(ph, Sx[ri]), ez));
            f2 = cneg(cadd(cmul(Sz0[ri], rx), cmul(Sx[ri], rz)));
        }
        out[r] = cadd(f1, f2);
    }
}

// Qc/Qh rows 0..2MF, and G = up*J - wq*I for the Pz product (ScatterVolume.cpp:823-881)
__global__ void q_kernel(const double2* __restrict__ V, const double2* __restrict__ beta, int MF,
                         const double* __restrict__ upk, const double* __restrict__ wqk, int Mx,
                         double2* __restrict__ Qc, double2* __restrict__ Qh, double2* __restrict__ Gc,
                         double2* __restrict__ Gh) {
    const int z = blockIdx.y;
    const int n4 = 4 * MF, n2 = 2 * MF, n3 = 3 * MF;
    const double2* v = V + (long long)z * n4 * n4;
    const double2* be = beta + (long long)z * n4;
    const long long tot = (long long)n2 * n2;   // 2MF rows x 2MF cols
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(t % n2), j = (int)(t / n2);
        const double2 bev = be[2 * j], bod = be[2 * j + 1];
        const double2* ce = v + (long long)(2 * j) * n4;
        const double2* co = v + (long long)(2 * j + 1) * n4;
        Qc[(long long)z * n3 * n2 + (long long)j * n3 + r] = cmul(ce[r], bev);
        Qh[(long long)z * n3 * n2 + (long long)j * n3 + r] = cmul(co[r], bod);
        if (r < MF) {
            // r is the Phi-order index qj*Mx + pj of the H rows
            const double up = upk[r % Mx], wq = wqk[r / Mx];
            const double2 I1 = cmul(ce[n2 + r], bev), J1 = cmul(ce[n2 + MF + r], bev);
            const double2 I2 = cmul(co[n2 + r], bod), J2 = cmul(co[n2 + MF + r], bod);
            Gc[(long long)z * MF * n2 + (long long)j * MF + r] = csub(cscale(J1, up), cscale(I1, wq));
            Gh[(long long)z * MF * n2 + (long long)j * MF + r] = csub(cscale(J2, up), cscale(I2, wq));
        }
    }
}

// KP (MF x MF): NIf[lin] with lin = ((indR+My/2)%My)*Mx + (indC+Mx/2)%Mx read
// as a linear index into the column-major My x Mx coefficients
// (ScatterVolume.cpp:867-875), scaled by -1/k.
__global__ void kp_kernel(const double2* __restrict__ Nif, int Mx, int My, double k, double2* __restrict__ KP) {
    const int z = blockIdx.y;
    const int MF = Mx * My;
    const long long tot = (long long)MF * MF;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(t % MF), c = (int)(t / MF);
        const int qi = r / Mx, pi_ = r % Mx, qj = c / Mx, pj = c % Mx;
        const int indR = (qi - qj + My) % My, indC = (pi_ - pj + Mx) % Mx;
        const int lin = ((indR + My / 2) % My) * Mx + (indC + Mx / 2) % Mx;
        KP[(long long)z * tot + t] = cscale(Nif[(long long)z * MF + lin], -1.0 / k);
    }
}

unsigned grid_for(long long tot, int tpb = 256) {
    long long b = (tot + tpb - 1) / tpb;
    if (b < 1) b = 1;
    if (b > 8192) b = 8192;
    return (unsigned)b;
}

template <typename T>
sc_status upload(cudaStream_t st, T* dst, const std::vector<T>& src) {
    if (src.empty()) return SC_OK;
    SC_CUDA_TRY(cudaMemcpyAsync(dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice, st));
    return SC_OK;
}

// slices / forcing of a precision code (SC_SWEEP_FP64, _MIXED, _CRT, _SLICES(s))
bool precision_slices(int precision, int* slices, bool* force, bool* crt) {
    *force = false;
    *crt = false;
    if (precision == SC_SWEEP_FP64) *slices = 0;
    else if (precision == SC_SWEEP_MIXED) *slices = 7;
    else if (precision == SC_SWEEP_CRT) {
        *slices = 7;
        *crt = true;
    } else if ((precision & ~0xFF) == 0x100 && (precision & 0xFF) >= 1 && (precision & 0xFF) <= 7) {
        *slices = precision & 0xFF;
        *force = true;
    } else
        return false;
    return true;
}

// C = A B (alpha 1, beta 0), strided batch: the FP64 tile when the engine has
// no digit slices (the reference-precision path), else the engine
sc_status product(cudaStream_t st, const GemmEngine& eng, int m, int n, int k, const double2* A, int lda, long long sA,
                  const double2* B, int ldb, long long sB, double2* C, int ldc, long long sC, int batch) {
    if (eng.slices == 0)
        return zgemm(st, m, n, k, make_double2(1.0, 0.0), A, lda, sA, B, ldb, sB, make_double2(0.0, 0.0), C, ldc, sC,
                     batch);
    GemmArgs g;
    g.m = m;
    g.n = n;
    g.k = k;
    g.A = A;
    g.lda = lda;
    g.sA = sA;
    g.B = B;
    g.ldb = ldb;
    g.sB = sB;
    g.C = C;
    g.ldc = ldc;
    g.sC = sC;
    return eng.run(st, g, batch);
}

}  // namespace

sc_status set_volume_precision(sc_context* ctx, int precision) {
    int sl;
    bool force, crt;
    if (!precision_slices(precision, &sl, &force, &crt)) {
        set_error("sc_volume_precision: unknown precision %d", precision);
        return SC_BADINPUT;
    }
    ctx->precision = precision;
    return SC_OK;
}

// ---------------------------------------------------------------- the plan
sc_status make_plan(const sc_volume_params* p, int Z, int S1, int S2, VolumePlan* plan) {
    if (!p || !plan || Z <= 0 || S1 <= 0 || S2 <= 0) {
        set_error("volume plan: bad sample shape (%d, %d, %d)", Z, S1, S2);
        return SC_BADINPUT;
    }
    if (!(p->lambda > 0.0) || !(p->size[0] > 0.0) || !(p->size[1] > 0.0) || !(p->size[2] > 0.0)) {
        set_error("volume plan: lambda and size must be positive");
        return SC_BADINPUT;
    }
    VolumePlan& P = *plan;
    P = VolumePlan();
    P.S1 = S1;
    P.S2 = S2;
    sc_volume_dims& D = P.dims;
    // direction and polarisation (ScatterVolume.cpp:575-583, FourierWave.h:32-39)
    double dn = std::sqrt(p->direction[0] * p->direction[0] + p->direction[1] * p->direction[1] +
                          p->direction[2] * p->direction[2]);
    if (!(dn > 0.0)) {
        set_error("volume plan: zero direction");
        return SC_BADINPUT;
    }
    double d[3] = {p->direction[0] / dn, p->direction[1] / dn, p->direction[2] / dn};
    cplx E[3] = {cplx(p->ex[0], p->ex[1]), cplx(p->ey[0], p->ey[1]), cplx(p->ez[0], p->ez[1])};
    cplx mag = std::sqrt(E[0] * E[0] + E[1] * E[1] + E[2] * E[2]);
    for (auto& e : E) e /= mag;
    auto cross = [](const cplx* a, const cplx* b, cplx* o) {
        o[0] = a[1] * b[2] - a[2] * b[1];
        o[1] = a[2] * b[0] - a[0] * b[2];
        o[2] = a[0] * b[1] - a[1] * b[0];
    };
    cplx dc[3] = {d[0], d[1], d[2]}, s[3], e2[3];
    cross(E, dc, s);
    cross(dc, s, e2);
    for (int i = 0; i < 3; ++i) {
        D.e_re[i] = e2[i].real();
        D.e_im[i] = e2[i].imag();
        D.dir[i] = d[i] * p->n[0];
    }
    D.k = 2 * PI_TRUNC / p->lambda;
    D.Z = Z;
    P.n_top = cplx(p->n[0], 0.0);
    P.n_bot = cplx(p->n[1], p->kappa);
    // z planes (ScatterVolume.cpp:162-168)
    P.z.resize(Z + 1);
    P.z[0] = p->z - p->size[2] / 2.0;
    for (int i = 1; i <= Z; ++i) P.z[i] = P.z[i - 1] + p->size[2] / Z;
    // orders (ScatterVolume.cpp:599-651)
    int M0 = S2, M1 = S1;
    if (p->ncoef == 1) {
        M0 = M1 = (int)std::sqrt((double)p->coef[0]);
    } else if (p->ncoef >= 2) {
        M0 = p->coef[0];
        M1 = p->coef[1];
    }
    const double lam = p->lambda, *sz = p->size, *n = p->n, *dir = D.dir;
    D.clamped = 0;
    if (std::pow((double)(M0 / 2) / sz[0] * lam + dir[0], 2) + std::pow((double)(M1 / 2) / sz[1] * lam + dir[1], 2) >=
        std::pow(n[0], 2)) {
        D.clamped = 1;
        if (M0 != 1 && M1 != 1) {
            if ((double)(M0 / 2) / sz[0] * lam + dir[0] > 0.71 * n[0]) M0 = (int)(0.707 * n[0] * 2 * sz[0] / lam) - 1;
            if ((double)(M1 / 2) / sz[1] * lam + dir[1] > 0.71 * n[0]) M1 = (int)(0.707 * n[1] * 2 * sz[1] / lam) - 1;
        }
        if (M0 == 1) {
            if ((double)(M1 / 2) / sz[1] * lam + std::fabs(dir[1]) >= n[0]) {
                M1 = (int)(n[1] * 2 * sz[1] / lam - 1e-10);
                if (M1 % 2 == 0) M1 -= 1;
            }
        }
        if (M1 == 1) {
            if ((double)(M0 / 2) / sz[1] * lam + std::fabs(dir[0]) >= n[0]) {
                M0 = (int)(n[0] * 2 * sz[0] / lam - 1e-10);
                if (M0 % 2 == 0) M0 -= 1;
            }
        }
    }
    if (M0 > S2) M0 = S2;
    if (M1 > S1) M1 = S1;
    if (M0 < 1 || M1 < 1) {
        set_error("volume plan: no Fourier orders left (Mx=%d, My=%d)", M0, M1);
        return SC_BADINPUT;
    }
    D.Mx = M0;
    D.My = M1;
    D.MF = M0 * M1;
    const int Mx = M0, My = M1, MF = D.MF;
    // lattice (FourierWave.h:319-334) and the Pz lattice (ScatterVolume.cpp:811-814)
    P.up.resize(Mx);
    P.wq.resize(My);
    P.UP.resize(Mx);
    P.WQ.resize(My);
    for (int i = 0; i < Mx; ++i) {
        double ps = (Mx == 1) ? (double)((Mx - 1) / 2) : -(double)(Mx / 2) + i * (((double)((Mx - 1) / 2) + (double)(Mx / 2)) / (Mx - 1));
        P.up[i] = 2 * PI_TRUNC * ps / sz[0] + dir[0] * D.k;
        P.UP[i] = 2.0 * ps * M_PI / sz[0];
    }
    for (int i = 0; i < My; ++i) {
        double qs = (My == 1) ? (double)((My - 1) / 2) : -(double)(My / 2) + i * (((double)((My - 1) / 2) + (double)(My / 2)) / (My - 1));
        P.wq[i] = 2 * PI_TRUNC * qs / sz[1] + dir[1] * D.k;
        P.WQ[i] = 2.0 * qs * M_PI / sz[1];
    }
    P.Sx.resize(MF);
    P.Sy.resize(MF);
    P.Sz0.resize(MF);
    P.Sz1.resize(MF);
    for (int pidx = 0; pidx < MF; ++pidx) {
        const int r = pidx % My, c = pidx / My;   // column-major (My x Mx) flattening
        cplx sx = P.up[c] / D.k, sy = P.wq[r] / D.k;
        P.Sx[pidx] = sx;
        P.Sy[pidx] = sy;
        P.Sz0[pidx] = std::sqrt(P.n_top * P.n_top - sx * sx - sy * sy);
        P.Sz1[pidx] = std::sqrt(P.n_bot * P.n_bot - sx * sx - sy * sy);
    }
    // incident spectrum (ScatterVolume.cpp:661-679): the transform of a constant
    // slice is its DC bin alone, placed wherever the crop tables put bin (0, 0);
    // --psf sets every order
    P.EF.assign(3 * MF, cplx(0.0, 0.0));
    std::vector<int> by, bx;
    crop_bins(S1, S2, My, Mx, by, bx);
    for (int c = 0; c < 3; ++c) {
        cplx e(D.e_re[c], D.e_im[c]);
        for (int j = 0; j < Mx; ++j)
            for (int i = 0; i < My; ++i)
                if (p->psf || (by[i] == 0 && bx[j] == 0)) P.EF[c * MF + i + j * My] = e;
    }
    return SC_OK;
}

// ---------------------------------------------------------------- the solve
namespace {

// per-solve state shared by the stages: plan, product engine and the small
// host-built device arrays (lattice, z planes, S vectors, EF)
struct VolumeRun {
    VolumePlan P;
    int Mx = 0, My = 0, MF = 0, n2 = 0, n4 = 0, n6 = 0, Z = 0;
    long long s2 = 0, s4 = 0;
    double k = 0.0;
    GemmEngine eng;
    const double *d_up = nullptr, *d_upk = nullptr, *d_wqk = nullptr, *d_z = nullptr, *d_kz0 = nullptr;
    double2* svec = nullptr;   // Sx, Sy, Sz0, Sz1, EF (7 MF)
};

sc_status volume_setup(sc_context* ctx, const sc_volume_params* p, int Z, int S1, int S2, cudaStream_t st,
                       VolumeRun& v) {
    SC_TRY(make_plan(p, Z, S1, S2, &v.P));
    const VolumePlan& P = v.P;
    v.Mx = P.dims.Mx;
    v.My = P.dims.My;
    v.MF = P.dims.MF;
    v.n2 = 2 * v.MF;
    v.n4 = 4 * v.MF;
    v.n6 = 6 * v.MF;
    v.Z = Z;
    v.s2 = (long long)v.n2 * v.n2;
    v.s4 = (long long)v.n4 * v.n4;
    v.k = P.dims.k;
    const int Mx = v.Mx, My = v.My, MF = v.MF;
    const double k = v.k;
    Workspace& ws = ctx->ws;
    for (int i = 0; i < 7; ++i)
        if (!ctx->ev[i]) SC_CUDA_TRY(cudaEventCreate(&ctx->ev[i]));
    // products of the transfer chain, the boundary block and Pz: FP64 tiles, or
    // the int8 engines under a mixed precision setting (the FFT, assembly,
    // Omega, the eigensolve, the eigenvectors and every LU stay FP64)
    precision_slices(ctx->precision, &v.eng.slices, &v.eng.force_int8, &v.eng.force_crt);
    v.eng.ws = &ws;
    if (v.eng.slices) {
        SC_TRY(ws.get(&v.eng.err, 1, WS_OZ_ERR, st));
        SC_CUDA_TRY(cudaMemsetAsync(v.eng.err, 0, sizeof(int), st));
    }
    double* lat = nullptr;     // up (Mx), wq (My), UPk (Mx), WQk (My), z (Z+1), k, z0
    const size_t nlat = (size_t)2 * (Mx + My) + Z + 3;
    SC_TRY(ws.get(&lat, nlat, WS_LAT, st));
    std::vector<double> hl(nlat);
    for (int i = 0; i < Mx; ++i) hl[i] = P.up[i];
    for (int i = 0; i < My; ++i) hl[Mx + i] = P.wq[i];
    for (int i = 0; i < Mx; ++i) hl[Mx + My + i] = P.UP[i] + P.dims.dir[0] * k;
    for (int i = 0; i < My; ++i) hl[2 * Mx + My + i] = P.WQ[i] + P.dims.dir[1] * k;
    for (int i = 0; i <= Z; ++i) hl[2 * (Mx + My) + i] = P.z[i];
    hl[2 * (Mx + My) + Z + 1] = k;
    hl[2 * (Mx + My) + Z + 2] = P.z[0];
    SC_TRY(upload(st, lat, hl));
    v.d_up = lat;
    v.d_upk = lat + Mx + My;
    v.d_wqk = lat + 2 * Mx + My;
    v.d_z = lat + 2 * (Mx + My);
    v.d_kz0 = v.d_z + Z + 1;
    SC_TRY(ws.get(&v.svec, (size_t)7 * MF, WS_EVAL_W, st));
    std::vector<cplx> hv;
    hv.reserve(7 * MF);
    hv.insert(hv.end(), P.Sx.begin(), P.Sx.end());
    hv.insert(hv.end(), P.Sy.begin(), P.Sy.end());
    hv.insert(hv.end(), P.Sz0.begin(), P.Sz0.end());
    hv.insert(hv.end(), P.Sz1.begin(), P.Sz1.end());
    hv.insert(hv.end(), P.EF.begin(), P.EF.end());
    SC_CUDA_TRY(cudaMemcpyAsync(v.svec, hv.data(), hv.size() * sizeof(cplx), cudaMemcpyHostToDevice, st));
    return SC_OK;
}

// device buffers of the layer stages, kept for the interior stage
struct LayerBufs {
    double2 *Nif = nullptr, *V = nullptr, *evl = nullptr, *dG = nullptr, *cG = nullptr, *Inv = nullptr;
    double2* Gcs = nullptr;     // the ordered chain product of the layers
    int* dinfo = nullptr;       // per-layer eigensolve status, then boundary LU status at [Zb]
};

// a3-a9 for layers [lb, le) of the sample: Fourier coefficients, B, C and
// Omega, eigenpairs, GD/GC and all GD_i^-1, and the ordered chain product
//   Gcs = T_{le-1} ... T_{lb},  T_i = GC_i GD_i^-1 = V_i diag(cG_i) GD_i^-1,
// in which layer 0 (when lb == 0) contributes GC_0 itself (ScatterVolume.cpp:
// 282-336 multiplies the same factors in sequence; here a pairwise tree).
// Events ev[1..4] mark the stage boundaries.
sc_status volume_layers(sc_context* ctx, VolumeRun& v, const double2* sample, int S1, int S2, int lb, int le,
                        cudaStream_t st, LayerBufs& b) {
    const int Zb = le - lb, MF = v.MF, n2 = v.n2, n4 = v.n4;
    const long long s2 = v.s2, s4 = v.s4;
    Workspace& ws = ctx->ws;
    // ---- a3: Fourier coefficients
    double2 *Nf, *R2, *Ri2;
    SC_TRY(ws.get(&Nf, (size_t)Zb * MF, WS_NF, st));
    SC_TRY(ws.get(&b.Nif, (size_t)Zb * MF, WS_NIF, st));
    SC_TRY(ws.get(&R2, (size_t)Zb * S1 * v.Mx, WS_TMP, st));
    SC_TRY(ws.get(&Ri2, (size_t)Zb * S1 * v.Mx, WS_TMP2, st));
    int* bins;
    SC_TRY(ws.get(&bins, (size_t)v.Mx + v.My, WS_BINS, st));
    SC_TRY(fft2_crop(st, sample + (long long)lb * S1 * S2, Zb, S1, S2, v.Mx, v.My, Nf, b.Nif, R2, Ri2, bins));
    SC_CUDA_TRY(cudaEventRecord(ctx->ev[1], st));

    // ---- a5: B, C blocks and Omega = B C
    double2 *Bm, *Cm, *Om;
    SC_TRY(ws.get(&Bm, (size_t)Zb * s2, WS_BMAT, st));
    SC_TRY(ws.get(&Cm, (size_t)Zb * s2, WS_CMAT, st));
    SC_TRY(ws.get(&Om, (size_t)Zb * s2, WS_OMEGA, st));
    SC_TRY(assemble_bc(st, Nf, b.Nif, Zb, v.Mx, v.My, v.d_up, v.k, Bm, Cm));
    SC_TRY(zgemm(st, n2, n2, n2, make_double2(1.0, 0.0), Bm, n2, s2, Cm, n2, s2, make_double2(0.0, 0.0), Om, n2,
                 s2, Zb));
    SC_CUDA_TRY(cudaEventRecord(ctx->ev[2], st));

    // ---- a7/a8: eigenpairs
    double2 *mu, *Wm, *CW;
    SC_TRY(ws.get(&mu, (size_t)Zb * n2, WS_MU, st));
    SC_TRY(ws.get(&Wm, (size_t)Zb * s2, WS_W, st));
    SC_TRY(ws.get(&CW, (size_t)Zb * s2, WS_CW, st));
    SC_TRY(ws.get(&b.V, (size_t)Zb * s4, WS_V, st));
    SC_TRY(ws.get(&b.evl, (size_t)Zb * n4, WS_EVL, st));
    SC_TRY(ws.get(&b.dinfo, (size_t)Zb + 4, WS_INFO, st));
    SC_CUDA_TRY(cudaMemsetAsync(b.dinfo, 0, sizeof(int) * (Zb + 4), st));
    SC_TRY(eig_batched(st, Om, n2, Zb, mu, Wm, b.dinfo, ws));
    SC_TRY(zgemm(st, n2, n2, n2, make_double2(1.0, 0.0), Cm, n2, s2, Wm, n2, s2, make_double2(0.0, 0.0), CW, n2,
                 s2, Zb));
    {
        dim3 g(grid_for(s4), Zb);
        build_v_kernel<<<g, 256, 0, st>>>(mu, Wm, CW, n2, b.V, b.evl);
        count_launch();
    }
    SC_TRY(normalize_columns(st, b.V, n4, n4, n4, s4, Zb));
    SC_CUDA_TRY(cudaEventRecord(ctx->ev[3], st));

    // ---- a9: GD/GC, explicit GD_i^-1 for all layers, and the chain product
    double2 *LU, *tree;
    int* piv;
    SC_TRY(ws.get(&b.dG, (size_t)Zb * n4, WS_TMP, st));
    SC_TRY(ws.get(&b.cG, (size_t)Zb * n4, WS_TMP2, st));
    SC_TRY(ws.get(&LU, (size_t)Zb * s4, WS_GD, st));
    SC_TRY(ws.get(&b.Inv, (size_t)Zb * s4, WS_INV, st));
    SC_TRY(ws.get(&piv, (size_t)Zb * n4, WS_PIV, st));
    SC_TRY(ws.get(&b.Gcs, (size_t)s4, WS_T, st));
    {
        dim3 g((n4 + 255) / 256, Zb);
        gdgc_scale_kernel<<<g, 256, 0, st>>>(b.evl, n4, Zb, v.d_z + lb, v.k, b.dG, b.cG);
        count_launch();
        dim3 g2(grid_for(s4), Zb);
        scale_cols_kernel<<<g2, 256, 0, st>>>(b.V, s4, b.dG, n4, n4, n4, LU, s4);
        count_launch();
    }
    SC_TRY(getrf(st, LU, n4, s4, n4, Zb, piv, nullptr));
    SC_TRY(set_identity(st, b.Inv, n4, s4, n4, Zb));
    SC_TRY(getrs(st, LU, n4, s4, n4, piv, b.Inv, n4, s4, n4, Zb));
    {
        // level 0 of the tree: M_i = T_{lb+i}; with lb == 0 the first is GC_0 = V_0 diag(cG_0)
        const int nt = Zb;
        SC_TRY(ws.get(&tree, (size_t)(nt + (nt + 1) / 2) * s4, WS_TREE, st));
        int first = 0;
        if (lb == 0) {
            scale_cols_kernel<<<dim3(grid_for(s4), 1), 256, 0, st>>>(b.V, s4, b.cG, n4, n4, n4, tree, s4);
            count_launch();
            first = 1;
        }
        if (first < Zb) {
            // rows of GD_i^-1 scaled by cG_i, into the spare half of the tree buffer, then T_i = V_i (.)
            double2* scaled = tree + (long long)nt * s4;
            for (int i0 = first; i0 < Zb; i0 += (nt + 1) / 2) {
                const int cnt = (Zb - i0) < (nt + 1) / 2 ? (Zb - i0) : (nt + 1) / 2;
                dim3 g(grid_for(s4), cnt);
                scale_rows_batched_kernel<<<g, 256, 0, st>>>(b.Inv + i0 * s4, s4, b.cG + (long long)i0 * n4, n4, n4,
                                                            n4, scaled, s4);
                count_launch();
                SC_TRY(product(st, v.eng, n4, n4, n4, b.V + i0 * s4, n4, s4, scaled, n4, s4, tree + i0 * s4, n4, s4,
                               cnt));
            }
        }
        // pairwise products M_{2j+1} M_{2j}, level by level (order preserved)
        double2* cur = tree;
        double2* nxt = tree + (long long)nt * s4;
        int cnt = nt;
        while (cnt > 1) {
            const int pairs = cnt / 2;
            SC_TRY(product(st, v.eng, n4, n4, n4, cur + s4, n4, 2 * s4, cur, n4, 2 * s4, nxt, n4, s4, pairs));
            if (cnt & 1)
                SC_CUDA_TRY(cudaMemcpyAsync(nxt + pairs * s4, cur + (cnt - 1) * s4, sizeof(double2) * s4,
                                            cudaMemcpyDeviceToDevice, st));
            cnt = pairs + (cnt & 1);
            double2* t = cur;
            cur = nxt;
            nxt = t;
        }
        SC_CUDA_TRY(cudaMemcpyAsync(b.Gcs, cur, sizeof(double2) * s4, cudaMemcpyDeviceToDevice, st));
    }
    SC_CUDA_TRY(cudaEventRecord(ctx->ev[4], st));
    return SC_OK;
}

// a10-a13 (ScatterVolume.cpp:339-466, 739): f3, Gc_static^-1 f3 (Gcs is
// factored in place), A6[2MF:, 3MF:] = GD_0 (.), the Gaussian rows, the
// incident right-hand side, and the LU solve; returns b6 = [R; T] (6 MF) and
// the boundary LU status word in *dinfo_lu
sc_status volume_boundary(sc_context* ctx, VolumeRun& v, double2* Gcs, const double2* GD0, int* dinfo_lu,
                          cudaStream_t st, double2** b6_out) {
    const int MF = v.MF, n4 = v.n4, n6 = v.n6;
    const long long s4 = v.s4;
    Workspace& ws = ctx->ws;
    double2 *F, *A6, *b6;
    int* piv6;
    SC_TRY(ws.get(&F, (size_t)n4 * 3 * MF, WS_F, st));
    SC_TRY(ws.get(&A6, (size_t)n6 * n6, WS_A6, st));
    SC_TRY(ws.get(&b6, (size_t)n6, WS_B6, st));
    SC_TRY(ws.get(&piv6, (size_t)n6 + n4, WS_PIV6, st));
    SC_TRY(boundary_f3(st, MF, v.svec, 0, F, 0, 1));
    SC_TRY(getrf(st, Gcs, n4, s4, n4, 1, piv6 + n6, nullptr));
    SC_TRY(getrs(st, Gcs, n4, s4, n4, piv6 + n6, F, n4, 0, 3 * MF, 1));
    SC_TRY(boundary_system(st, MF, v.svec, 0, v.d_kz0, A6, 0, b6, 0, 1));
    SC_TRY(product(st, v.eng, n4, 3 * MF, n4, GD0, n4, s4, F, n4, 0, A6 + (long long)3 * MF * n6 + 2 * MF, n6, 0,
                   1));
    SC_TRY(getrf(st, A6, n6, 0, n6, 1, piv6, dinfo_lu));
    SC_TRY(getrs(st, A6, n6, 0, n6, piv6, b6, n6, 0, 1, 1));
    *b6_out = b6;
    return SC_OK;
}

sc_status volume_engine_status(VolumeRun& v) {
    if (!v.eng.slices) return SC_OK;
    int herr = 0;
    SC_CUDA_TRY(cudaMemcpy(&herr, v.eng.err, sizeof(int), cudaMemcpyDeviceToHost));
    if (herr) {
        set_error("volume solve: tensor-core pipeline wait timed out (stage %d)", herr);
        return SC_CUDA_ERROR;
    }
    return SC_OK;
}

}  // namespace

sc_status volume_solve(sc_context* ctx, const sc_volume_params* p, const double2* sample, int Z, int S1,
                       int S2, double2* x_out, double2* evl_out, double2* Qc_out, double2* Qh_out,
                       int* info_host, cudaStream_t st) {
    VolumeRun v;
    SC_TRY(volume_setup(ctx, p, Z, S1, S2, st, v));
    SC_CUDA_TRY(cudaEventRecord(ctx->ev[0], st));
    const int Mx = v.Mx, My = v.My, MF = v.MF, n2 = v.n2, n4 = v.n4;
    const long long s4 = v.s4;
    const double k = v.k;
    Workspace& ws = ctx->ws;
    LayerBufs b;
    SC_TRY(volume_layers(ctx, v, sample, S1, S2, 0, Z, st, b));

    // ---- a10-a13: boundary system and its solve, with GD_0 = V_0 diag(dG_0)
    double2* X;
    SC_TRY(ws.get(&X, (size_t)s4, WS_T2, st));
    scale_cols_kernel<<<dim3(grid_for(s4), 1), 256, 0, st>>>(b.V, s4, b.dG, n4, n4, n4, X, s4);
    count_launch();
    double2* b6;
    SC_TRY(volume_boundary(ctx, v, b.Gcs, X, b.dinfo + Z, st, &b6));
    if (x_out) SC_CUDA_TRY(cudaMemcpyAsync(x_out, b6, sizeof(double2) * v.n6, cudaMemcpyDeviceToDevice, st));
    SC_CUDA_TRY(cudaEventRecord(ctx->ev[5], st));

    // ---- a14/a15: beta chain, Q, Pz
    const double2 *dSx = v.svec, *dSy = v.svec + MF, *dSz0 = v.svec + 2 * MF, *dEF = v.svec + 4 * MF;
    if (!p->external && (Qc_out || Qh_out)) {
        double2 *beta, *tv, *gpart;
        SC_TRY(ws.get(&gpart, zgemv_part_size(n4, n4, 1) + 2 * (size_t)n4, WS_GEMV, st));
        SC_TRY(ws.get(&beta, (size_t)Z * n4 + 2 * n4, WS_BETA, st));
        tv = beta + (long long)Z * n4;
        double2* rhs = tv + n4;
        beta0_rhs_kernel<<<grid_for(n4), 256, 0, st>>>(MF, dSx, dSy, dSz0, dEF, b6, k, v.P.z[0], rhs);
        count_launch();
        // beta_0 = GD_0^-1 (f1 EF + f2 R);  beta_i = GD_i^-1 V_{i-1} (cG_{i-1} .* beta_{i-1})
        SC_TRY(zgemv(st, n4, n4, make_double2(1.0, 0.0), b.Inv, n4, s4, rhs, 0, make_double2(0.0, 0.0), beta, 0, 1,
                     gpart));
        for (int i = 1; i < Z; ++i) {
            scale_cols_kernel<<<dim3(grid_for(n4), 1), 256, 0, st>>>(beta + (long long)(i - 1) * n4, 0,
                                                                      b.cG + (long long)(i - 1) * n4, 0, 1, n4,
                                                                      rhs, 0);
            count_launch();
            SC_TRY(zgemv(st, n4, n4, make_double2(1.0, 0.0), b.V + (i - 1) * s4, n4, s4, rhs, 0,
                         make_double2(0.0, 0.0), tv, 0, 1, gpart));
            SC_TRY(zgemv(st, n4, n4, make_double2(1.0, 0.0), b.Inv + i * s4, n4, s4, tv, 0, make_double2(0.0, 0.0),
                         beta + (long long)i * n4, 0, 1, gpart));
        }
        double2 *Gc, *Gh, *KP;
        SC_TRY(ws.get(&Gc, (size_t)Z * MF * n2 * 2, WS_PZ, st));
        Gh = Gc + (long long)Z * MF * n2;
        SC_TRY(ws.get(&KP, (size_t)Z * MF * MF, WS_OMEGA, st));
        double2* Qc = Qc_out;
        double2* Qh = Qh_out;
        const long long sq = (long long)3 * MF * n2;
        {
            dim3 g(grid_for((long long)n2 * n2), Z);
            q_kernel<<<g, 256, 0, st>>>(b.V, beta, MF, v.d_upk, v.d_wqk, Mx, Qc, Qh, Gc, Gh);
            count_launch();
        }
        if (!p->npz) {
            dim3 g(grid_for((long long)MF * MF), Z);
            kp_kernel<<<g, 256, 0, st>>>(b.Nif, Mx, My, k, KP);
            count_launch();
            SC_TRY(product(st, v.eng, MF, n2, MF, KP, MF, (long long)MF * MF, Gc, MF, (long long)MF * n2, Qc + n2,
                           3 * MF, sq, Z));
            SC_TRY(product(st, v.eng, MF, n2, MF, KP, MF, (long long)MF * MF, Gh, MF, (long long)MF * n2, Qh + n2,
                           3 * MF, sq, Z));
        } else {
            for (int z = 0; z < Z; ++z) {
                SC_CUDA_TRY(cudaMemset2DAsync(Qc + z * sq + n2, sizeof(double2) * 3 * MF, 0, sizeof(double2) * MF,
                                              n2, st));
                SC_CUDA_TRY(cudaMemset2DAsync(Qh + z * sq + n2, sizeof(double2) * 3 * MF, 0, sizeof(double2) * MF,
                                              n2, st));
            }
        }
    }
    if (evl_out) SC_CUDA_TRY(cudaMemcpyAsync(evl_out, b.evl, sizeof(double2) * Z * n4, cudaMemcpyDeviceToDevice, st));
    SC_CUDA_TRY(cudaEventRecord(ctx->ev[6], st));

    // ---- status: eig info per layer + boundary LU info
    std::vector<int> hinfo(Z + 4, 0);
    SC_CUDA_TRY(cudaMemcpyAsync(hinfo.data(), b.dinfo, sizeof(int) * (Z + 4), cudaMemcpyDeviceToHost, st));
    SC_CUDA_TRY(cudaStreamSynchronize(st));
    for (int i = 0; i < 6; ++i) {
        float ms = 0.f;
        SC_CUDA_TRY(cudaEventElapsedTime(&ms, ctx->ev[i], ctx->ev[i + 1]));
        ctx->stage_ms[i] = ms;
    }
    {
        float ms = 0.f;
        SC_CUDA_TRY(cudaEventElapsedTime(&ms, ws.ev_hqr[0], ws.ev_hqr[1]));
        ctx->stage_ms[6] = ms;
        SC_CUDA_TRY(cudaEventElapsedTime(&ms, ctx->ev[0], ctx->ev[6]));
        ctx->stage_ms[7] = ms;
    }
    SC_TRY(volume_engine_status(v));
    int first = 0;
    for (int i = 0; i < Z && !first; ++i) first = hinfo[i];
    if (info_host) *info_host = first ? first : hinfo[Z];
    if (first) {
        set_error("eigensolve did not converge (layer status %d)", first);
        return SC_NOCONVERGE;
    }
    if (hinfo[Z]) {
        set_error("boundary system is singular (zero pivot in column %d)", hinfo[Z] - 1);
        return SC_SINGULAR;
    }
    return SC_OK;
}

sc_status volume_chain_block(sc_context* ctx, const sc_volume_params* p, const double2* sample, int Z, int S1,
                             int S2, int lb, int le, double2* P_out, double2* GD0_out, int* info_host,
                             cudaStream_t st) {
    if (lb < 0 || le > Z || lb >= le) {
        set_error("sc_volume_chain_block: layer range [%d, %d) outside [0, %d)", lb, le, Z);
        return SC_BADINPUT;
    }
    VolumeRun v;
    SC_TRY(volume_setup(ctx, p, Z, S1, S2, st, v));
    SC_CUDA_TRY(cudaEventRecord(ctx->ev[0], st));
    LayerBufs b;
    SC_TRY(volume_layers(ctx, v, sample, S1, S2, lb, le, st, b));
    SC_CUDA_TRY(cudaMemcpyAsync(P_out, b.Gcs, sizeof(double2) * v.s4, cudaMemcpyDeviceToDevice, st));
    if (GD0_out) {
        if (lb != 0) {
            set_error("sc_volume_chain_block: GD_0 belongs to the block that starts at layer 0");
            return SC_BADINPUT;
        }
        scale_cols_kernel<<<dim3(grid_for(v.s4), 1), 256, 0, st>>>(b.V, v.s4, b.dG, v.n4, v.n4, v.n4, GD0_out,
                                                                    v.s4);
        count_launch();
        SC_CHECK_LAUNCH("chain block GD_0");
    }
    const int Zb = le - lb;
    std::vector<int> hinfo(Zb, 0);
    SC_CUDA_TRY(cudaMemcpyAsync(hinfo.data(), b.dinfo, sizeof(int) * Zb, cudaMemcpyDeviceToHost, st));
    SC_CUDA_TRY(cudaStreamSynchronize(st));
    SC_TRY(volume_engine_status(v));
    int first = 0;
    for (int i = 0; i < Zb && !first; ++i) first = hinfo[i];
    if (info_host) *info_host = first;
    if (first) {
        set_error("eigensolve did not converge (layer status %d)", first);
        return SC_NOCONVERGE;
    }
    return SC_OK;
}

sc_status volume_boundary_solve(sc_context* ctx, const sc_volume_params* p, int Z, int S1, int S2,
                                const double2* Gcs_in, const double2* GD0, double2* x_out, int* info_host,
                                cudaStream_t st) {
    VolumeRun v;
    SC_TRY(volume_setup(ctx, p, Z, S1, S2, st, v));
    double2* Gcs;
    int* dinfo;
    SC_TRY(ctx->ws.get(&Gcs, (size_t)v.s4, WS_T, st));
    SC_TRY(ctx->ws.get(&dinfo, 4, WS_INFO, st));
    SC_CUDA_TRY(cudaMemsetAsync(dinfo, 0, sizeof(int) * 4, st));
    SC_CUDA_TRY(cudaMemcpyAsync(Gcs, Gcs_in, sizeof(double2) * v.s4, cudaMemcpyDeviceToDevice, st));
    double2* b6;
    SC_TRY(volume_boundary(ctx, v, Gcs, GD0, dinfo, st, &b6));
    SC_CUDA_TRY(cudaMemcpyAsync(x_out, b6, sizeof(double2) * v.n6, cudaMemcpyDeviceToDevice, st));
    int h = 0;
    SC_CUDA_TRY(cudaMemcpyAsync(&h, dinfo, sizeof(int), cudaMemcpyDeviceToHost, st));
    SC_CUDA_TRY(cudaStreamSynchronize(st));
    SC_TRY(volume_engine_status(v));
    if (info_host) *info_host = h;
    if (h) {
        set_error("boundary system is singular (zero pivot in column %d)", h - 1);
        return SC_SINGULAR;
    }
    return SC_OK;
}

}  // namespace sc
