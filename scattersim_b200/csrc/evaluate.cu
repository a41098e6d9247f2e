// Plane-wave tables and the field evaluator.
//
// volume_waves builds, on the device, the wave list the reference writes into
// the CoupledWaveStructure (ScatterVolume.cpp:907-987) in cw_unpack order
// (cpuEvaluator.cpp:61-102): Pi, then per boundary l its Pr list and its Pt
// list, each wave already wound to the origin (E0 <- E0 exp(-i kz z_l)).
// Region l of the evaluator is [begin[l], end[l]) of that table.
//
// cw_evaluate is the sum of gpuEvaluator.cu:28-68 over an arbitrary point
// list: region lookup #{z >= z_l - zeps}, then E = sum E0 exp(i k.r).
//   precision 0: float64 throughout;
//   precision 1: float32 amplitudes and accumulation, the phase k.r formed and
//                reduced modulo 2 pi in float64 before the float32 sincos.
// Waves are staged through shared memory in tiles of 256; a block's points
// are consecutive so that, for grid slices, a warp shares one region.
#include "common.cuh"
#include "kernels.cuh"

namespace sc {

namespace {
constexpr int ET = 256;

struct WaveSrc {
    int MF, Z, external, ez_mode;
    const double2 *Sx, *Sy, *Sz0, *Sz1, *EF, *x, *evl, *Qc, *Qh;
    const double* zpl;
    double k, ntop, nbot;
};

// one entry of the table: kind 0 incident, 1 reflected, 2 transmitted (order
// p), 3 internal (order p, mode jj of `layer`'s list `parity`, e[] already
// holding the mode's field from Q); returns E0 wound to the origin and k
__device__ __forceinline__ void wave_entry(const WaveSrc& s, int kind, long long p, long long jj, int layer,
                                           int parity, double zl, double2 (&e)[3], double2 (&kv)[3]) {
    const int MF = s.MF;
    kv[0] = cscale(s.Sx[p], s.k);
    kv[1] = cscale(s.Sy[p], s.k);
    if (kind == 0) {
        kv[2] = cscale(s.Sz0[p], s.k);
        e[0] = s.EF[p];
        e[1] = s.EF[MF + p];
        e[2] = s.EF[2 * MF + p];
    } else if (kind == 1) {
        kv[2] = cscale(s.Sz0[p], -s.k * s.ntop);
        e[0] = s.x[p];
        e[1] = s.x[MF + p];
        e[2] = s.x[2 * MF + p];
    } else if (kind == 2) {
        kv[2] = cscale(s.Sz1[p], s.k * s.nbot);
        e[0] = s.x[3 * MF + p];
        e[1] = s.x[4 * MF + p];
        e[2] = s.x[5 * MF + p];
    } else {
        kv[2] = cscale(s.evl[(long long)layer * 4 * MF + 2 * jj + parity], s.k);
    }
    if (s.ez_mode == 1) {
        // E_z from transversality, as the .cw reader rebuilds it
        e[2] = cneg(cdiv(cadd(cmul(kv[0], e[0]), cmul(kv[1], e[1])), kv[2]));
    }
    if (kind != 0) {
        // wind(0, 0, -z_l): E0 *= exp(i kz (-z_l))
        double2 ph = cexp(cmul(make_double2(0.0, 1.0), cscale(kv[2], -zl)));
        for (int c = 0; c < 3; ++c) e[c] = cmul(e[c], ph);
    }
}

// Table layout (cw_unpack order): Pi (MF) | Pr_0 (MF) | layer 0 parity 0,
// layer 0 parity 1, ..., layer Z-1 parity 1 (2 MF x MF waves each, order p
// major, mode jj minor; absent with --external) | Pt_Z (MF).
// The three boundary lists: one thread per wave; Pt_Z starts at t_base
// (2 MF + the internal lists in the full table, 2 MF in a compact one).
__global__ void waves_boundary_kernel(WaveSrc s, long long t_base, double2* __restrict__ E0,
                                      double2* __restrict__ K) {
    const int MF = s.MF;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < 3 * MF; t += gridDim.x * blockDim.x) {
        const int kind = t / MF;
        const long long p = t - (long long)kind * MF;
        const long long w = (kind == 2) ? t_base + p : t;
        const double zl = (kind == 1) ? s.zpl[0] : (kind == 2) ? s.zpl[s.Z] : 0.0;
        double2 e[3], kv[3];
        wave_entry(s, kind, p, 0, -1, 0, zl, e, kv);
        for (int c = 0; c < 3; ++c) {
            E0[w * 3 + c] = e[c];
            K[w * 3 + c] = kv[c];
        }
    }
}

// The internal lists, one block per tile of 16 modes x 32 orders of one list
// (grid z = 2 layer + parity): the mode fields are read from Q along the
// order index (contiguous in Q) into shared memory, and the table is written
// along the mode index (contiguous in the table), both coalesced.
constexpr int WJ = 16, WP = 32;
__global__ void __launch_bounds__(256) waves_internal_kernel(WaveSrc s, double2* __restrict__ E0,
                                                             double2* __restrict__ K) {
    __shared__ double2 sq[3][WJ][WP + 1];
    const int MF = s.MF, n2 = 2 * MF, n3 = 3 * MF;
    const int q = blockIdx.z, layer = q >> 1, parity = q & 1;
    const int j0 = blockIdx.x * WJ, p0 = blockIdx.y * WP;
    const double2* Q = (parity ? s.Qh : s.Qc) + (long long)layer * n3 * n2;
    for (int e = threadIdx.x; e < 3 * WJ * WP; e += blockDim.x) {
        const int c = e / (WJ * WP), r = (e / WP) % WJ, pp = e % WP;
        const int jj = j0 + r, p = p0 + pp;
        sq[c][r][pp] = (jj < n2 && p < MF) ? Q[(long long)jj * n3 + c * MF + p] : make_double2(0.0, 0.0);
    }
    __syncthreads();
    const double zl = s.zpl[layer + parity];
    const long long w0 = 2LL * MF + (long long)q * n2 * MF;
    for (int e = threadIdx.x; e < WJ * WP; e += blockDim.x) {
        const int jl = e % WJ, pl = e / WJ;
        const int jj = j0 + jl, p = p0 + pl;
        if (jj >= n2 || p >= MF) continue;
        double2 ev[3] = {sq[0][jl][pl], sq[1][jl][pl], sq[2][jl][pl]}, kv[3];
        wave_entry(s, 3, p, jj, layer, parity, zl, ev, kv);
        const long long w = w0 + (long long)p * n2 + jj;
        for (int c = 0; c < 3; ++c) {
            E0[w * 3 + c] = ev[c];
            K[w * 3 + c] = kv[c];
        }
    }
}

template <int PREC>
__global__ void __launch_bounds__(ET)
eval_kernel(const double2* __restrict__ E0, const double2* __restrict__ K, const double* __restrict__ zl,
            const int* __restrict__ begin, const int* __restrict__ end, int layers, double zeps,
            const double* __restrict__ pts, long long np, double2* __restrict__ out) {
    __shared__ double2 sE[ET * 3];
    __shared__ double2 sK[ET * 3];
    __shared__ int s_lo, s_hi;
    const long long pidx = (long long)blockIdx.x * ET + threadIdx.x;
    const bool active = pidx < np;
    double px = 0.0, py = 0.0, pz = 0.0;
    int reg = 0;
    if (active) {
        px = pts[pidx * 3 + 0];
        py = pts[pidx * 3 + 1];
        pz = pts[pidx * 3 + 2];
        for (int l = 0; l < layers; ++l)
            if (pz >= zl[l] - zeps) reg = l + 1;
    }
    // block-wide range of regions
    if (threadIdx.x == 0) {
        s_lo = 1 << 30;
        s_hi = -1;
    }
    __syncthreads();
    if (active) {
        atomicMin(&s_lo, reg);
        atomicMax(&s_hi, reg);
    }
    __syncthreads();
    const int rlo = s_lo, rhi = s_hi;
    double2 a0 = make_double2(0, 0), a1 = make_double2(0, 0), a2 = make_double2(0, 0);
    float2 f0 = make_float2(0, 0), f1 = make_float2(0, 0), f2 = make_float2(0, 0);
    const double TWO_PI = 6.283185307179586;
    for (int r = rlo; r <= rhi; ++r) {
        const int wb = begin[r], we = end[r];
        for (int t0 = wb; t0 < we; t0 += ET) {
            const int nt = (we - t0) < ET ? (we - t0) : ET;
            __syncthreads();
            for (int q = threadIdx.x; q < nt * 3; q += ET) {
                sE[q] = E0[(long long)t0 * 3 + q];
                sK[q] = K[(long long)t0 * 3 + q];
            }
            __syncthreads();
            if (active && reg == r) {
                for (int q = 0; q < nt; ++q) {
                    const double2 kx = sK[q * 3], ky = sK[q * 3 + 1], kz = sK[q * 3 + 2];
                    const double phr = kx.x * px + ky.x * py + kz.x * pz;
                    const double phi = kx.y * px + ky.y * py + kz.y * pz;
                    if (PREC == 0) {
                        double s, c;
                        sincos(phr, &s, &c);
                        const double amp = exp(-phi);
                        const double2 ph = make_double2(amp * c, amp * s);
                        a0 = cfma(sE[q * 3], ph, a0);
                        a1 = cfma(sE[q * 3 + 1], ph, a1);
                        a2 = cfma(sE[q * 3 + 2], ph, a2);
                    } else {
                        const double red = phr - TWO_PI * rint(phr * (1.0 / TWO_PI));
                        float s, c;
                        sincosf((float)red, &s, &c);
                        const float amp = expf((float)(-phi));
                        const float2 ph = make_float2(amp * c, amp * s);
                        const double2 e0 = sE[q * 3], e1 = sE[q * 3 + 1], e2 = sE[q * 3 + 2];
                        f0 = fcfma(make_float2((float)e0.x, (float)e0.y), ph, f0);
                        f1 = fcfma(make_float2((float)e1.x, (float)e1.y), ph, f1);
                        f2 = fcfma(make_float2((float)e2.x, (float)e2.y), ph, f2);
                    }
                }
            }
        }
    }
    if (active) {
        if (PREC == 0) {
            out[pidx * 3 + 0] = a0;
            out[pidx * 3 + 1] = a1;
            out[pidx * 3 + 2] = a2;
        } else {
            out[pidx * 3 + 0] = make_double2(f0.x, f0.y);
            out[pidx * 3 + 1] = make_double2(f1.x, f1.y);
            out[pidx * 3 + 2] = make_double2(f2.x, f2.y);
        }
    }
}
}  // namespace

sc_status volume_waves_launch(cudaStream_t st, int MF, int Z, const double2* svec, const double2* x,
                              const double2* evl, const double2* Qc, const double2* Qh, const double* zpl,
                              double k, double ntop, double nbot, int external, int ez_mode, long long nw,
                              double2* E0, double2* K) {
    const long long internal = external ? 0 : 2LL * Z * (2LL * MF * MF);
    if (nw != 3LL * MF + internal) {
        set_error("volume_waves: table of %lld waves, expected %lld", nw, 3LL * MF + internal);
        return SC_BADINPUT;
    }
    WaveSrc s{MF, Z, external, ez_mode, svec, svec + MF, svec + 2 * MF, svec + 3 * MF, svec + 4 * MF,
              x, evl, Qc, Qh, zpl, k, ntop, nbot};
    waves_boundary_kernel<<<(3 * MF + 255) / 256, 256, 0, st>>>(s, 2LL * MF + internal, E0, K);
    count_launch();
    if (internal > 0) {
        if (2LL * Z > 65535) {
            set_error("volume_waves: too many layers (%d)", Z);
            return SC_BADINPUT;
        }
        waves_internal_kernel<<<dim3((2 * MF + WJ - 1) / WJ, (MF + WP - 1) / WP, 2 * Z), 256, 0, st>>>(s, E0, K);
        count_launch();
    }
    SC_CHECK_LAUNCH("volume_waves");
    return SC_OK;
}

// the compact table of the three boundary lists only: Pi | Pr_0 | Pt_Z (3 MF waves)
sc_status volume_boundary_waves_launch(cudaStream_t st, int MF, int Z, const double2* svec, const double2* x,
                                       const double* zpl, double k, double ntop, double nbot, int external,
                                       int ez_mode, double2* E0, double2* K) {
    WaveSrc s{MF, Z, external, ez_mode, svec, svec + MF, svec + 2 * MF, svec + 3 * MF, svec + 4 * MF,
              x, nullptr, nullptr, nullptr, zpl, k, ntop, nbot};
    waves_boundary_kernel<<<(3 * MF + 255) / 256, 256, 0, st>>>(s, 2LL * MF, E0, K);
    count_launch();
    SC_CHECK_LAUNCH("volume_boundary_waves");
    return SC_OK;
}

sc_status cw_evaluate_launch(cudaStream_t st, const double2* E0, const double2* K, const double* zl,
                             const int* begin, const int* end, int layers, double zeps, const double* pts,
                             long long np, double2* out, int precision) {
    if (np <= 0) return SC_OK;
    long long blocks = (np + ET - 1) / ET;
    if (precision == 0)
        eval_kernel<0><<<(unsigned)blocks, ET, 0, st>>>(E0, K, zl, begin, end, layers, zeps, pts, np, out);
    else
        eval_kernel<1><<<(unsigned)blocks, ET, 0, st>>>(E0, K, zl, begin, end, layers, zeps, pts, np, out);
    count_launch();
    SC_CHECK_LAUNCH("cw_evaluate");
    return SC_OK;
}

}  // namespace sc
