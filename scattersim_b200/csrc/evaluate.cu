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

__global__ void waves_kernel(int MF, int Z, const double2* __restrict__ Sx, const double2* __restrict__ Sy,
                             const double2* __restrict__ Sz0, const double2* __restrict__ Sz1,
                             const double2* __restrict__ EF, const double2* __restrict__ x,
                             const double2* __restrict__ evl, const double2* __restrict__ Qc,
                             const double2* __restrict__ Qh, const double* __restrict__ zpl, double k, double ntop,
                             double nbot, int external, int ez_mode, long long nw, double2* __restrict__ E0,
                             double2* __restrict__ K) {
    const int n2 = 2 * MF, n3 = 3 * MF, n4 = 4 * MF;
    const long long internal = (long long)n2 * MF;   // waves per internal list
    for (long long w = (long long)blockIdx.x * blockDim.x + threadIdx.x; w < nw;
         w += (long long)gridDim.x * blockDim.x) {
        // locate the wave: Pi | (Pr_0, Pt_0) | (Pr_1, Pt_1) | ... | (Pr_Z, Pt_Z)
        long long o = w;
        double2 e[3], kv[3];
        double zl = 0.0;
        int kind = -1, layer = -1, parity = 0;
        long long idx = 0;
        if (o < MF) {
            kind = 0;  // incident
            idx = o;
        } else {
            o -= MF;
            for (int l = 0; l <= Z && kind < 0; ++l) {
                long long npr = (l == 0) ? MF : (external ? 0 : internal);
                long long npt = (l == Z) ? MF : (external ? 0 : internal);
                if (o < npr) {
                    if (l == 0) kind = 1;  // reflected
                    else { kind = 3; layer = l - 1; parity = 1; }
                    idx = o;
                    zl = zpl[l];
                } else if (o < npr + npt) {
                    o -= npr;
                    if (l == Z) kind = 2;  // transmitted
                    else { kind = 3; layer = l; parity = 0; }
                    idx = o;
                    zl = zpl[l];
                } else {
                    o -= npr + npt;
                }
            }
        }
        if (kind <= 2) {
            const long long p = idx;
            kv[0] = cscale(Sx[p], k);
            kv[1] = cscale(Sy[p], k);
            if (kind == 0) {
                kv[2] = cscale(Sz0[p], k);
                e[0] = EF[p];
                e[1] = EF[MF + p];
                e[2] = EF[2 * MF + p];
            } else if (kind == 1) {
                kv[2] = cscale(Sz0[p], -k * ntop);
                e[0] = x[p];
                e[1] = x[MF + p];
                e[2] = x[2 * MF + p];
            } else {
                kv[2] = cscale(Sz1[p], k * nbot);
                e[0] = x[3 * MF + p];
                e[1] = x[4 * MF + p];
                e[2] = x[5 * MF + p];
            }
        } else {
            const long long p = idx / n2, jj = idx % n2;
            kv[0] = cscale(Sx[p], k);
            kv[1] = cscale(Sy[p], k);
            kv[2] = cscale(evl[(long long)layer * n4 + 2 * jj + parity], k);
            const double2* Q = (parity ? Qh : Qc) + (long long)layer * n3 * n2 + jj * n3;
            e[0] = Q[p];
            e[1] = Q[MF + p];
            e[2] = Q[2 * MF + p];
        }
        if (ez_mode == 1) {
            // E_z from transversality, as the .cw reader rebuilds it
            e[2] = cneg(cdiv(cadd(cmul(kv[0], e[0]), cmul(kv[1], e[1])), kv[2]));
        }
        if (kind != 0) {
            // wind(0, 0, -z_l): E0 *= exp(i kz (-z_l))
            double2 ph = cexp(cmul(make_double2(0.0, 1.0), cscale(kv[2], -zl)));
            for (int c = 0; c < 3; ++c) e[c] = cmul(e[c], ph);
        }
        for (int c = 0; c < 3; ++c) {
            E0[w * 3 + c] = e[c];
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
    long long blocks = (nw + 255) / 256;
    if (blocks > 16384) blocks = 16384;
    if (blocks < 1) blocks = 1;
    waves_kernel<<<(unsigned)blocks, 256, 0, st>>>(MF, Z, svec, svec + MF, svec + 2 * MF, svec + 3 * MF,
                                                   svec + 4 * MF, x, evl, Qc, Qh, zpl, k, ntop, nbot, external,
                                                   ez_mode, nw, E0, K);
    count_launch();
    SC_CHECK_LAUNCH("volume_waves");
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
