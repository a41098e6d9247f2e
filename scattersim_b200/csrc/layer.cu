// Homogeneous multilayer and single-interface solves, batched over the plane
// waves of a focused beam.
//
// scatterlayer (ScatterLayer.cpp:110-420) solves, for every incident plane
// wave of a beam, one 6L x 6L linear system (boundary conditions :152-165,
// Gaussian constraints :167-184, tangential E/H continuity :186-232) and turns
// its solution into a reflected and a transmitted wave per boundary
// (mat2waves :234-266, wound by -z_l :404-409).  scatterplane
// (ScatterPlane.cpp:81-264) is the same solve with one interface.  The beam
// itself is tira::planewave::SolidAnglePolar (a polar grid of directions about
// the centre wave, every wave carrying the centre wave's record pair scaled by
// its solid angle sin(theta) dtheta dphi); that rule, and the record frame
// of the coupled-wave file, are pinned by reproducing data/psf.cw and x64/a.cw.
//
// beam_polar_kernel: one thread per wave.
// layer_solve_kernel: one warp per wave.  The warp builds the system in its
// own slice of shared memory (row stride n + 1 so that a quarter warp's
// 16-byte column accesses fall in distinct banks), factors it by LU with
// partial pivoting (pivot search by warp arg-max; in the trailing update each
// lane owns a column and walks rows), back-substitutes and writes the wound
// waves.  The reference uses colPivHouseholderQr; both are backward stable on
// this square system and agree to rounding.  A wave whose system has an exact zero pivot gets
// SC_SINGULAR in its status word.
#include <cmath>
#include <vector>

#include "context.cuh"

namespace sc {

namespace {

constexpr int LAYER_MAX = 15;           // 6L x 6L system of one wave fits one warp's shared memory
constexpr int LS_WARPS = 4;             // warps (waves) per CTA, fewer when the system is large

struct BeamArgs {
    double Rc[9];         // frame of the centre wave (row-major)
    double2 a, b;         // centre wave's record pair
    double kmag, beta, dth, dph, f[3];
    int N0, count;
};

// tira frame of a real direction kh (unit): minimal rotation z -> kh; columns 0 and 1
__device__ __forceinline__ void frame_cols(const double kh[3], double c0[3], double c1[3]) {
    const double ax0 = -kh[1], ax1 = kh[0];
    const double s2 = ax0 * ax0 + ax1 * ax1;
    if (s2 < 1e-30) {
        const double sg = kh[2] > 0.0 ? 1.0 : -1.0;
        c0[0] = 1.0; c0[1] = 0.0; c0[2] = 0.0;
        c1[0] = 0.0; c1[1] = sg;  c1[2] = 0.0;
        return;
    }
    const double f = (1.0 - kh[2]) / s2;
    c0[0] = 1.0 - f * ax1 * ax1; c0[1] = f * ax0 * ax1;       c0[2] = -ax1;
    c1[0] = f * ax0 * ax1;       c1[1] = 1.0 - f * ax0 * ax0; c1[2] = ax0;
}

__global__ void beam_polar_kernel(BeamArgs p, double* __restrict__ kout, double2* __restrict__ Eout) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= p.count) return;
    const int i = t % p.N0, j = t / p.N0;
    const double th = p.beta + i * p.dth, ph = j * p.dph;
    double st, ct, sp, cp;
    sincos(th, &st, &ct);
    sincos(ph, &sp, &cp);
    const double loc[3] = {st * cp, st * sp, ct};
    double kh[3];
    for (int r = 0; r < 3; ++r) kh[r] = p.Rc[3 * r] * loc[0] + p.Rc[3 * r + 1] * loc[1] + p.Rc[3 * r + 2] * loc[2];
    const double nrm = sqrt(kh[0] * kh[0] + kh[1] * kh[1] + kh[2] * kh[2]);
    for (int r = 0; r < 3; ++r) kh[r] /= nrm;
    double c0[3], c1[3];
    frame_cols(kh, c0, c1);
    const double w = st * p.dth * p.dph;
    // wound to the focal point: E0 exp(-i k . f)
    const double kf = p.kmag * (kh[0] * p.f[0] + kh[1] * p.f[1] + kh[2] * p.f[2]);
    double sf, cf;
    sincos(-kf, &sf, &cf);
    const double2 ph0 = make_double2(w * cf, w * sf);
    for (int r = 0; r < 3; ++r) {
        kout[3 * (long long)t + r] = p.kmag * kh[r];
        const double2 e = cadd(cscale(p.a, c0[r]), cscale(p.b, c1[r]));
        Eout[3 * (long long)t + r] = cmul(e, ph0);
    }
}

struct LayerArgs {
    const double2* ri;    // L complex refractive indices
    const double* z;      // L - 1 boundaries
    double kvac, n0;
    int L, count;
};

__device__ __forceinline__ double2 expi(double2 w) {   // exp(i w), w complex
    return cexp(make_double2(-w.y, w.x));
}

__global__ void layer_solve_kernel(LayerArgs p, const double* __restrict__ kin, const double2* __restrict__ Ein,
                                   double2* __restrict__ rE, double2* __restrict__ rk, double2* __restrict__ tE,
                                   double2* __restrict__ tk, int* __restrict__ status) {
    extern __shared__ double2 sm[];
    const int L = p.L, n = 6 * L, ld = n + 1;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const long long g = (long long)blockIdx.x * (blockDim.x >> 5) + warp;
    if (g >= p.count) return;
    double2* A = sm + (size_t)warp * (n * ld + n + L);
    double2* b = A + n * ld;
    double2* sz = b + n;
    // direction (ScatterLayer getDirection), s = d n0 for sz (InitSz :133-148)
    double d[3] = {kin[3 * g], kin[3 * g + 1], kin[3 * g + 2]};
    const double dn = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    for (int c = 0; c < 3; ++c) d[c] /= dn;
    const double s0 = d[0] * p.n0, s1 = d[1] * p.n0;
    for (int l = lane; l < L; l += 32) {
        const double2 r = p.ri[l];
        sz[l] = csqrt(make_double2(r.x * r.x - r.y * r.y - s0 * s0 - s1 * s1, 2.0 * r.x * r.y));
    }
    for (int e = lane; e < n * ld + n; e += 32) A[e] = make_double2(0.0, 0.0);
    __syncwarp();
    // one row per lane (row-major A[r * ld + c]); unknown idx(l, dir, c) = 6 l + 3 dir + c
    const double2 one = make_double2(1.0, 0.0), mone = make_double2(-1.0, 0.0);
    const int rowG = 6, rowB = 6 + 2 * (L - 1);
    for (int r = lane; r < n; r += 32) {
        double2* row = A + (size_t)r * ld;
        if (r < 3) {                                   // transmitted wave of layer 0 = incident (:152-160)
            row[r] = one;
            b[r] = Ein[3 * g + r];
        } else if (r < 6) {                            // no reflected wave in the last layer (:162-164)
            row[6 * (L - 1) + 3 + (r - 3)] = one;
        } else if (r < rowG + (L - 1)) {               // reflected Gaussian constraint, layer l (:170-176)
            const int l = r - rowG;
            row[6 * l + 3] = make_double2(d[0], 0.0);
            row[6 * l + 4] = make_double2(d[1], 0.0);
            row[6 * l + 5] = cneg(sz[l]);
        } else if (r < rowB) {                         // transmitted Gaussian constraint, layer l (:178-183)
            const int l = r - (rowG + L - 2);
            row[6 * l + 0] = make_double2(d[0], 0.0);
            row[6 * l + 1] = make_double2(d[1], 0.0);
            row[6 * l + 2] = sz[l];
        } else {                                       // continuity at boundary l (:186-232)
            const int q = r - rowB, l = q >> 2, sub = q & 3;
            const double zn = (l == 0) ? p.z[0] : p.z[l] - p.z[l - 1];
            const double zp = (l == L - 2) ? 0.0 : p.z[l] - p.z[l + 1];
            const double2 et = expi(cscale(sz[l], p.kvac * zn));
            const double2 er = expi(cscale(sz[l + 1], -p.kvac * zp));
            const int tl = 6 * l, rl = 6 * l + 3, tn = 6 * (l + 1), rn = 6 * (l + 1) + 3;
            const double2 dx = make_double2(d[0], 0.0), dy = make_double2(d[1], 0.0);
            if (sub == 0) {
                row[tl + 0] = et; row[rl + 0] = one; row[tn + 0] = mone; row[rn + 0] = cneg(er);
            } else if (sub == 1) {
                row[tl + 1] = et; row[rl + 1] = one; row[tn + 1] = mone; row[rn + 1] = cneg(er);
            } else if (sub == 2) {
                row[tl + 2] = cmul(dy, et);
                row[tl + 1] = cneg(cmul(sz[l], et));
                row[rl + 2] = dy;
                row[rl + 1] = sz[l];
                row[tn + 2] = cneg(dy);
                row[tn + 1] = sz[l + 1];
                row[rn + 2] = cneg(cmul(dy, er));
                row[rn + 1] = cneg(cmul(sz[l + 1], er));
            } else {
                row[tl + 0] = cmul(sz[l], et);
                row[tl + 2] = cneg(cmul(dx, et));
                row[rl + 0] = cneg(sz[l]);
                row[rl + 2] = cneg(dx);
                row[tn + 0] = cneg(sz[l + 1]);
                row[tn + 2] = dx;
                row[rn + 0] = cmul(sz[l + 1], er);
                row[rn + 2] = cmul(dx, er);
            }
        }
    }
    __syncwarp();
    // LU with partial pivoting (row swaps of whole rows, multipliers kept in place)
    int singular = 0;
    for (int j = 0; j < n; ++j) {
        double bv = -1.0;
        int bi = n;
        for (int i = j + lane; i < n; i += 32) {
            const double v = cabs1(A[i * ld + j]);
            if (v > bv) { bv = v; bi = i; }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const double ov = __shfl_xor_sync(0xffffffffu, bv, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            if (ov > bv || (ov == bv && oi < bi)) { bv = ov; bi = oi; }
        }
        if (!(bv > 0.0)) {                             // zero (or NaN) column: uniform over the warp
            singular = 1;
            break;
        }
        if (bi != j) {
            for (int c = lane; c < n; c += 32) {
                const double2 t = A[j * ld + c];
                A[j * ld + c] = A[bi * ld + c];
                A[bi * ld + c] = t;
            }
            if (lane == 0) {
                const double2 t = b[j];
                b[j] = b[bi];
                b[bi] = t;
            }
        }
        __syncwarp();
        // multipliers: one reciprocal of the pivot per step
        const double2 rpiv = cdiv(make_double2(1.0, 0.0), A[j * ld + j]);
        for (int i = j + 1 + lane; i < n; i += 32) A[i * ld + j] = cmul(A[i * ld + j], rpiv);
        __syncwarp();
        // trailing update A(i, c) -= A(i, j) A(j, c), i, c > j: a lane keeps its column's
        // pivot-row entry in registers and walks rows; with m <= 32 columns the warp
        // is split into 32 / m row groups (one division per step, none per element)
        const int m = n - j - 1;
        if (m > 0 && m <= 32) {
            const int groups = 32 / m, cl = lane % m, r0 = lane / m;
            if (r0 < groups) {
                const int c = j + 1 + cl;
                const double2 najc = cneg(A[j * ld + c]);
#pragma unroll 4
                for (int i = j + 1 + r0; i < n; i += groups) A[i * ld + c] = cfma(A[i * ld + j], najc, A[i * ld + c]);
            }
        } else if (m > 32) {
            for (int c = j + 1 + lane; c < n; c += 32) {
                const double2 najc = cneg(A[j * ld + c]);
#pragma unroll 4
                for (int i = j + 1; i < n; ++i) A[i * ld + c] = cfma(A[i * ld + j], najc, A[i * ld + c]);
            }
        }
        for (int i = j + 1 + lane; i < n; i += 32) b[i] = csub(b[i], cmul(A[i * ld + j], b[j]));
        __syncwarp();
    }
    if (!singular) {
        for (int j = n - 1; j >= 0; --j) {
            const double2 xj = cdiv(b[j], A[j * ld + j]);
            __syncwarp();
            if (lane == 0) b[j] = xj;
            for (int i = lane; i < j; i += 32) b[i] = csub(b[i], cmul(A[i * ld + j], xj));
            __syncwarp();
        }
    }
    // mat2waves (:240-266) wound by -z_l (:404-409)
    const int nb = L - 1;
    for (int t = lane; t < 3 * nb; t += 32) {
        const int l = t / 3, c = t % 3;
        const long long o = (g * nb + l) * 3 + c;
        const double kxy = (c == 0 ? s0 : s1) * p.kvac;
        const double2 krz = cscale(sz[l], -p.kvac), ktz = cscale(sz[l + 1], p.kvac);
        rk[o] = c < 2 ? make_double2(kxy, 0.0) : krz;
        tk[o] = c < 2 ? make_double2(kxy, 0.0) : ktz;
        if (singular) {
            rE[o] = make_double2(0.0, 0.0);
            tE[o] = make_double2(0.0, 0.0);
        } else {
            rE[o] = cmul(b[6 * l + 3 + c], expi(cscale(krz, -p.z[l])));
            tE[o] = cmul(b[6 * (l + 1) + c], expi(cscale(ktz, -p.z[l])));
        }
    }
    if (lane == 0 && status) status[g] = singular ? SC_SINGULAR : SC_OK;
}

size_t layer_smem_per_wave(int L) {
    const size_t n = 6 * (size_t)L;
    return (n * (n + 1) + n + L) * sizeof(double2);
}

}  // namespace

sc_status beam_polar(cudaStream_t st, double alpha, double beta, int N0, int N1, const double* kc,
                     const double2* ec, const double* focus, double* kout, double2* Eout, int* count) {
    if (!kc || !ec || !kout || !Eout || !count || N0 <= 0 || N1 <= 0 || !std::isfinite(alpha) ||
        !std::isfinite(beta)) {
        set_error("beam_polar: bad argument");
        return SC_BADINPUT;
    }
    const double kmag = std::sqrt(kc[0] * kc[0] + kc[1] * kc[1] + kc[2] * kc[2]);
    if (!(kmag > 0.0) || !std::isfinite(kmag)) {
        set_error("beam_polar: zero or non-finite centre wave vector");
        return SC_BADINPUT;
    }
    BeamArgs p{};
    const double kh[3] = {kc[0] / kmag, kc[1] / kmag, kc[2] / kmag};
    // the centre frame (same rule as frame_cols, all three columns)
    const double ax0 = -kh[1], ax1 = kh[0], s2 = ax0 * ax0 + ax1 * ax1;
    double Rc[3][3];
    if (s2 < 1e-30) {
        const double sg = kh[2] > 0.0 ? 1.0 : -1.0;
        const double I[3][3] = {{1, 0, 0}, {0, sg, 0}, {0, 0, sg}};
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) Rc[r][c] = I[r][c];
    } else {
        const double f = (1.0 - kh[2]) / s2;
        const double R[3][3] = {{1.0 - f * ax1 * ax1, f * ax0 * ax1, ax1},
                                {f * ax0 * ax1, 1.0 - f * ax0 * ax0, -ax0},
                                {-ax1, ax0, kh[2]}};
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) Rc[r][c] = R[r][c];
    }
    for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c) p.Rc[3 * r + c] = Rc[r][c];
    // record pair of the centre wave: first two components of Rc^T e
    p.a = make_double2(0.0, 0.0);
    p.b = make_double2(0.0, 0.0);
    for (int r = 0; r < 3; ++r) {
        p.a = cadd(p.a, cscale(ec[r], Rc[r][0]));
        p.b = cadd(p.b, cscale(ec[r], Rc[r][1]));
    }
    p.kmag = kmag;
    p.f[0] = focus ? focus[0] : 0.0;
    p.f[1] = focus ? focus[1] : 0.0;
    p.f[2] = focus ? focus[2] : 0.0;
    if (alpha == 0.0 || (long long)N0 * N1 == 1) {
        // the single centre wave (ScatterLayer.cpp:378-379, ScatterPlane.cpp:215-216)
        p.N0 = 1;
        p.count = 1;
        p.beta = 0.0;
        p.dth = 0.0;
        p.dph = 0.0;
        std::vector<double> hk(kc, kc + 3);
        const double kf = kc[0] * p.f[0] + kc[1] * p.f[1] + kc[2] * p.f[2];
        const double2 ph = make_double2(std::cos(-kf), std::sin(-kf));
        std::vector<double2> he(3);
        for (int r = 0; r < 3; ++r) he[r] = cmul(ec[r], ph);
        SC_CUDA_TRY(cudaMemcpyAsync(kout, hk.data(), 3 * sizeof(double), cudaMemcpyHostToDevice, st));
        SC_CUDA_TRY(cudaMemcpyAsync(Eout, he.data(), 3 * sizeof(double2), cudaMemcpyHostToDevice, st));
        SC_CUDA_TRY(cudaStreamSynchronize(st));
        *count = 1;
        return SC_OK;
    }
    if ((long long)N0 * N1 > (1LL << 30)) {
        set_error("beam_polar: %d x %d samples is too many", N0, N1);
        return SC_BADINPUT;
    }
    p.N0 = N0;
    p.count = N0 * N1;
    p.beta = beta;
    p.dth = (alpha - beta) / N0;
    p.dph = 2.0 * M_PI / N1;
    beam_polar_kernel<<<(p.count + 255) / 256, 256, 0, st>>>(p, kout, Eout);
    count_launch();
    SC_CHECK_LAUNCH("beam_polar");
    *count = p.count;
    return SC_OK;
}

sc_status layer_solve(sc_context* ctx, int L, const double* n, const double* kappa, const double* z, double lambda,
                      int count, const double* kin, const double2* Ein, double2* rE, double2* rk, double2* tE,
                      double2* tk, int* status, cudaStream_t st) {
    if (L < 1 || L > LAYER_MAX || !n || (L > 1 && (!kappa || !z)) || count < 0 || !(lambda > 0.0) ||
        !std::isfinite(lambda)) {
        set_error("layer_solve: bad argument (layers %d, at most %d)", L, LAYER_MAX);
        return SC_BADINPUT;
    }
    if (count == 0) return SC_OK;
    if (!kin || !Ein || (L > 1 && (!rE || !rk || !tE || !tk))) {
        set_error("layer_solve: null device buffer");
        return SC_BADINPUT;
    }
    for (int l = 0; l < L; ++l)
        if (!std::isfinite(n[l]) || (l > 0 && !std::isfinite(kappa[l - 1]))) {
            set_error("layer_solve: non-finite refractive index in layer %d", l);
            return SC_BADINPUT;
        }
    for (int l = 0; l + 1 < L; ++l)
        if (!std::isfinite(z[l])) {
            set_error("layer_solve: non-finite boundary %d", l);
            return SC_BADINPUT;
        }
    // per-launch parameters: ri (L complex), z (L - 1), statuses when the caller passes none
    std::vector<double2> hri(L);
    hri[0] = make_double2(n[0], 0.0);                           // ScatterLayer.cpp:116-118
    for (int l = 1; l < L; ++l) hri[l] = make_double2(n[l], kappa[l - 1]);
    double2* dri = nullptr;
    SC_TRY(ctx->ws.get(&dri, (size_t)L + (L + 1) / 2, WS_LAYER, st));
    double* dz = reinterpret_cast<double*>(dri + L);
    SC_CUDA_TRY(cudaMemcpyAsync(dri, hri.data(), sizeof(double2) * L, cudaMemcpyHostToDevice, st));
    if (L > 1) SC_CUDA_TRY(cudaMemcpyAsync(dz, z, sizeof(double) * (L - 1), cudaMemcpyHostToDevice, st));
    int* dstat = status;
    if (!dstat) SC_TRY(ctx->ws.get(&dstat, (size_t)count, WS_LAYER_STATUS, st));
    LayerArgs p;
    p.ri = dri;
    p.z = dz;
    p.kvac = 2.0 * M_PI / lambda;                               // ScatterLayer.cpp:351
    p.n0 = n[0];
    p.L = L;
    p.count = count;
    const size_t per = layer_smem_per_wave(L);
    int warps = LS_WARPS;
    while (warps > 1 && per * warps > 96 * 1024) --warps;
    const size_t smem = per * warps;
    if (smem > 48 * 1024)
        SC_CUDA_TRY(cudaFuncSetAttribute(layer_solve_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const unsigned blocks = (unsigned)((count + warps - 1) / warps);
    layer_solve_kernel<<<blocks, 32 * warps, smem, st>>>(p, kin, Ein, rE, rk, tE, tk, dstat);
    count_launch();
    SC_CHECK_LAUNCH("layer_solve");
    std::vector<int> hs(count);
    SC_CUDA_TRY(cudaMemcpyAsync(hs.data(), dstat, sizeof(int) * count, cudaMemcpyDeviceToHost, st));
    SC_CUDA_TRY(cudaStreamSynchronize(st));
    for (int i = 0; i < count; ++i)
        if (hs[i] != SC_OK) {
            set_error("layer_solve: wave %d has a singular system", i);
            return SC_SINGULAR;
        }
    return SC_OK;
}

}  // namespace sc
