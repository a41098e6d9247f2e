// The field of a solved volume on a regular grid, in factorised form.
//
// The evaluator sum E(r) = sum_w E0_w exp(i k_w.r) over the waves of r's
// region (gpuEvaluator.cu:28-68) has, for a volume solution, the structure of
// the coupled-wave expansion: every wave of Fourier order p = (px, py) has the
// same transverse wave vector (kx_px, ky_py) (ScatterVolume.cpp:469-493,
// 907-987), and the region depends on z only.  On a grid x_i, y_j, z_b:
//   H_c[b](px, py) = sum over the region's waves of order p of E0_c exp(i kz z_b)
//   U_c[b](px, y_j) = sum_py exp(i ky_py y_j) H_c[b](px, py)
//   E_c(x_i, y_j, z_b) = sum_px exp(i kx_px x_i) U_c[b](px, y_j)
// which is the same sum regrouped: #waves x Nz exponentials plus two small
// products per plane, in place of #waves x Nx Ny Nz exponentials.  The wave
// table (and so every convention of the .cw waves: kz n factors, winding, the
// region test with zeps) is the one sc_volume_waves builds; the transverse
// wave numbers are read from it.  All arithmetic is FP64; the output is
// complex128 or complex64.
#include <algorithm>
#include <vector>

#include "common.cuh"
#include "context.cuh"
#include "kernels.cuh"

namespace sc {

sc_status volume_boundary_waves_launch(cudaStream_t st, int MF, int Z, const double2* svec, const double2* x,
                                       const double* zpl, double k, double ntop, double nbot, int external,
                                       int ez_mode, double2* E0, double2* K);

namespace {

constexpr int FH_THREADS = 128;
constexpr int FE_THREADS = 128;
constexpr int FE_MAXM = 64;    // orders along x the grid evaluator accepts
constexpr int FE_YCHUNK = 8;

struct FieldGeom {
    int MF, Mx, My, Z, external;
    int Nx, Ny, Nz;
    double x0, y0, z0, dx, dy, dz, zeps;
};

// transverse wave numbers from the table's incident list (order p = py + My px):
// kx[px] from the wave of order My px, ky[py] from the wave of order py
__global__ void field_k_kernel(FieldGeom g, const double2* __restrict__ K, double* __restrict__ kx,
                               double* __restrict__ ky) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < g.Mx) kx[t] = K[(long long)(g.My * t) * 3 + 0].x;
    if (t < g.My) ky[t] = K[(long long)t * 3 + 1].x;
}

// Ex[i + Nx px] = exp(i kx_px x_i), Ey[py + My j] = exp(i ky_py y_j)
__global__ void field_tables_kernel(FieldGeom g, const double* __restrict__ kx, const double* __restrict__ ky,
                                    double2* __restrict__ Ex, double2* __restrict__ Ey) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long nex = (long long)g.Nx * g.Mx, ney = (long long)g.My * g.Ny;
    if (t < nex) {
        const int i = (int)(t % g.Nx), px = (int)(t / g.Nx);
        double s, c;
        sincos(kx[px] * (g.x0 + g.dx * i), &s, &c);
        Ex[t] = make_double2(c, s);
    } else if (t < nex + ney) {
        const long long u = t - nex;
        const int py = (int)(u % g.My), j = (int)(u / g.My);
        double s, c;
        sincos(ky[py] * (g.y0 + g.dy * j), &s, &c);
        Ey[u] = make_double2(c, s);
    }
}

// H[b][c][px + Mx py]: one block per (order p, plane b); the region's lists
// are located from begin[] and the list layout of the wave table
__global__ void __launch_bounds__(FH_THREADS) field_h_kernel(FieldGeom g, const double2* __restrict__ E0,
                                                             const double2* __restrict__ K,
                                                             const double* __restrict__ zl,
                                                             double2* __restrict__ H) {
    __shared__ double2 red[3][FH_THREADS];
    const int p = blockIdx.x, b = blockIdx.y;
    const int MF = g.MF;
    const double z = g.z0 + g.dz * b;
    int l = 0;
    for (int i = 0; i <= g.Z; ++i)
        if (z >= zl[i] - g.zeps) l = i + 1;
    // the interior regions' planes are field_hq_kernel's (no waves with --external: H = 0)
    if (l >= 1 && l <= g.Z && !g.external) return;
    // lists of region l in the compact table Pi | Pr_0 | Pt_Z (one wave per order)
    long long s0 = (l == 0) ? 0 : (l == g.Z + 1) ? 2LL * MF : -1, s1 = (l == 0) ? MF : -1;
    const long long m0 = 1, m1 = 1;
    double2 acc[3] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
    for (int list = 0; list < 2; ++list) {
        const long long s = list ? s1 : s0, m = list ? m1 : m0;
        if (s < 0) continue;
        for (long long j = threadIdx.x; j < m; j += FH_THREADS) {
            const long long w = s + (long long)p * m + j;
            const double2 kz = K[w * 3 + 2];
            // exp(i kz z) with complex kz
            const double mag = exp(-kz.y * z);
            double sn, cs;
            sincos(kz.x * z, &sn, &cs);
            const double2 ph = make_double2(mag * cs, mag * sn);
#pragma unroll
            for (int c = 0; c < 3; ++c) acc[c] = cfma(E0[w * 3 + c], ph, acc[c]);
        }
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) red[c][threadIdx.x] = acc[c];
    __syncthreads();
    for (int s = FH_THREADS / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s)
#pragma unroll
            for (int c = 0; c < 3; ++c) red[c][threadIdx.x] = cadd(red[c][threadIdx.x], red[c][threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x < 3) {
        const int px = p / g.My, py = p % g.My;
        H[((long long)b * 3 + threadIdx.x) * MF + px + (long long)g.Mx * py] = red[threadIdx.x][0];
    }
}

// Order sums of the interior planes straight from the layers' mode fields,
// without the wave table: for plane b inside layer l,
//   H[b][c][p] = sum over modes jj of Qc_l[jj][c][p] exp(i kz0_jj (z_b - z_l))
//                                     + Qh_l[jj][c][p] exp(i kz1_jj (z_b - z_{l+1}))
// (kz_jj = k evl_l[2 jj + parity]; E_z rebuilt by transversality with
// ez_mode 1) -- the sum field_h_kernel forms over the table's two internal
// lists of the plane's region, each wave being Q wound by exp(-i kz z_l).
// A block takes 32 orders (a warp's lanes: Q is contiguous in the order
// index), up to HQ_NPL planes of one layer and one of HQ_JS slices of the
// modes; its 4 warps split the slice, the phases of a chunk of modes are
// shared through shared memory, and the slices' partial sums are added in
// a fixed order by field_hq_sum_kernel.
constexpr int HQ_P = 32, HQ_W = 4, HQ_NPL = 4, HQ_JC = 64, HQ_JS = 8;
struct PlaneGroup {
    int layer, first, count;   // planes plane_idx[first .. first + count) lie in `layer`
};

__device__ __forceinline__ int h_index(const FieldGeom& g, int p) { return p / g.My + g.Mx * (p % g.My); }

__global__ void __launch_bounds__(HQ_W * 32) field_hq_kernel(FieldGeom g, double k, const double2* __restrict__ Sx,
                                                              const double2* __restrict__ Sy,
                                                              const double2* __restrict__ evl,
                                                              const double2* __restrict__ Qc,
                                                              const double2* __restrict__ Qh,
                                                              const double* __restrict__ zpl,
                                                              const PlaneGroup* __restrict__ groups,
                                                              const int* __restrict__ plane_idx, int ez_mode,
                                                              double2* __restrict__ Hp) {
    __shared__ double2 ph[HQ_NPL][2][HQ_JC];
    __shared__ double2 rk[2][HQ_JC];
    __shared__ double2 red[HQ_W][HQ_NPL][3][HQ_P];
    const int MF = g.MF, n2 = 2 * MF, n3 = 3 * MF;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int p = blockIdx.x * HQ_P + lane;
    const PlaneGroup grp = groups[blockIdx.y];
    const int layer = grp.layer, np = grp.count;
    const int per = (n2 + HQ_JS - 1) / HQ_JS;
    const int jbeg = blockIdx.z * per, jend = min(n2, jbeg + per);
    const double2* qc = Qc + (long long)layer * n3 * n2;
    const double2* qh = Qh + (long long)layer * n3 * n2;
    const double zl0 = zpl[layer], zl1 = zpl[layer + 1];
    double zb[HQ_NPL];
#pragma unroll
    for (int pl = 0; pl < HQ_NPL; ++pl) zb[pl] = (pl < np) ? g.z0 + g.dz * plane_idx[grp.first + pl] : 0.0;
    double2 kx = make_double2(0.0, 0.0), ky = make_double2(0.0, 0.0);
    if (p < MF) {
        kx = cscale(Sx[p], k);
        ky = cscale(Sy[p], k);
    }
    double2 acc[HQ_NPL][3];
#pragma unroll
    for (int pl = 0; pl < HQ_NPL; ++pl)
#pragma unroll
        for (int c = 0; c < 3; ++c) acc[pl][c] = make_double2(0.0, 0.0);
    for (int j0 = jbeg; j0 < jend; j0 += HQ_JC) {
        const int nj = min(HQ_JC, jend - j0);
        __syncthreads();
        for (int t = threadIdx.x; t < 2 * nj; t += blockDim.x) {
            const int par = t / nj, jl = t - par * nj;
            const double2 kz = cscale(evl[(long long)layer * 4 * MF + 2 * (j0 + jl) + par], k);
            const double zr = par ? zl1 : zl0;
#pragma unroll
            for (int pl = 0; pl < HQ_NPL; ++pl)
                ph[pl][par][jl] = (pl < np) ? cexp(cmul(make_double2(0.0, 1.0), cscale(kz, zb[pl] - zr)))
                                            : make_double2(0.0, 0.0);
            if (ez_mode == 1) rk[par][jl] = cdiv(make_double2(1.0, 0.0), kz);
        }
        __syncthreads();
        if (p < MF) {
            for (int jl = warp; jl < nj; jl += HQ_W) {
                const long long o = (long long)(j0 + jl) * n3 + p;
                double2 ec[3] = {qc[o], qc[o + MF], qc[o + 2 * MF]};
                double2 eh[3] = {qh[o], qh[o + MF], qh[o + 2 * MF]};
                if (ez_mode == 1) {
                    ec[2] = cneg(cmul(cadd(cmul(kx, ec[0]), cmul(ky, ec[1])), rk[0][jl]));
                    eh[2] = cneg(cmul(cadd(cmul(kx, eh[0]), cmul(ky, eh[1])), rk[1][jl]));
                }
#pragma unroll
                for (int pl = 0; pl < HQ_NPL; ++pl) {
                    if (pl < np) {
                        const double2 p0 = ph[pl][0][jl], p1 = ph[pl][1][jl];
#pragma unroll
                        for (int c = 0; c < 3; ++c) acc[pl][c] = cfma(eh[c], p1, cfma(ec[c], p0, acc[pl][c]));
                    }
                }
            }
        }
    }
#pragma unroll
    for (int pl = 0; pl < HQ_NPL; ++pl)
#pragma unroll
        for (int c = 0; c < 3; ++c) red[warp][pl][c][lane] = acc[pl][c];
    __syncthreads();
    if (warp == 0 && p < MF) {
        for (int pl = 0; pl < np; ++pl) {
            const long long b = plane_idx[grp.first + pl];
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                double2 s = red[0][pl][c][lane];
                for (int w = 1; w < HQ_W; ++w) s = cadd(s, red[w][pl][c][lane]);
                Hp[(((long long)blockIdx.z * g.Nz + b) * 3 + c) * MF + h_index(g, p)] = s;
            }
        }
    }
}

// H of the interior planes = the sum of the HQ_JS mode slices, in order
__global__ void field_hq_sum_kernel(FieldGeom g, const int* __restrict__ plane_idx, int nint,
                                    const double2* __restrict__ Hp, double2* __restrict__ H) {
    const long long per = 3LL * g.MF, tot = (long long)nint * per;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < tot; t += (long long)gridDim.x * blockDim.x) {
        const long long b = plane_idx[t / per], r = t % per;
        double2 s = Hp[b * per + r];
        for (int q = 1; q < HQ_JS; ++q) s = cadd(s, Hp[((long long)q * g.Nz + b) * per + r]);
        H[b * per + r] = s;
    }
}

// U[b][c][px + Mx j] = sum_py H[b][c][px + Mx py] Ey[py + My j]
__global__ void field_u_kernel(FieldGeom g, const double2* __restrict__ H, const double2* __restrict__ Ey,
                               double2* __restrict__ U) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long per = (long long)g.Mx * g.Ny;
    const int bc = blockIdx.y;                     // b * 3 + c
    if (t >= per) return;
    const int px = (int)(t % g.Mx), j = (int)(t / g.Mx);
    const double2* h = H + (long long)bc * g.MF + px;
    const double2* e = Ey + (long long)g.My * j;
    double2 acc = make_double2(0.0, 0.0);
    for (int py = 0; py < g.My; ++py) acc = cfma(h[(long long)g.Mx * py], e[py], acc);
    U[(long long)bc * per + t] = acc;
}

// out[((b Ny + j) Nx + i) 3 + c] = sum_px Ex[i + Nx px] U[b][c][px + Mx j]; a
// thread owns one x_i (its Ex row in registers) and walks the y rows, the
// CTA staging FE_YCHUNK columns of U at a time
template <typename OUT, int MAXM>
__global__ void __launch_bounds__(FE_THREADS) field_e_kernel(FieldGeom g, const double2* __restrict__ Ex,
                                                             const double2* __restrict__ U, OUT* __restrict__ out) {
    __shared__ double2 su[FE_YCHUNK][3][MAXM];
    const int b = blockIdx.y;
    const int i = blockIdx.x * FE_THREADS + threadIdx.x;
    const bool active = i < g.Nx;
    const int Mx = g.Mx;
    double2 ex[MAXM];
#pragma unroll
    for (int px = 0; px < MAXM; ++px)
        ex[px] = (active && px < Mx) ? Ex[i + (long long)g.Nx * px] : make_double2(0.0, 0.0);
    const long long per = (long long)Mx * g.Ny;
    // this CTA's share of the y rows (blockIdx.z of gridDim.z, in whole chunks)
    const int chunks = (g.Ny + FE_YCHUNK - 1) / FE_YCHUNK;
    const int cper = (chunks + gridDim.z - 1) / gridDim.z;
    const int jbeg = blockIdx.z * cper * FE_YCHUNK;
    const int jend = min(g.Ny, jbeg + cper * FE_YCHUNK);
    for (int j0 = jbeg; j0 < jend; j0 += FE_YCHUNK) {
        const int nj = min(FE_YCHUNK, jend - j0);
        __syncthreads();
        for (int t = threadIdx.x; t < nj * 3 * Mx; t += FE_THREADS) {
            const int px = t % Mx, c = (t / Mx) % 3, jj = t / (3 * Mx);
            su[jj][c][px] = U[((long long)b * 3 + c) * per + px + (long long)Mx * (j0 + jj)];
        }
        __syncthreads();
        if (!active) continue;
        // two rows at a time: six independent complex accumulations per thread
        for (int jj = 0; jj < nj; jj += 2) {
            const int jb = (jj + 1 < nj) ? jj + 1 : jj;
            double2 e[2][3];
#pragma unroll
            for (int r = 0; r < 2; ++r)
#pragma unroll
                for (int c = 0; c < 3; ++c) e[r][c] = make_double2(0.0, 0.0);
#pragma unroll
            for (int px = 0; px < MAXM; ++px) {
                if (px < Mx) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        e[0][c] = cfma(ex[px], su[jj][c][px], e[0][c]);
                        e[1][c] = cfma(ex[px], su[jb][c][px], e[1][c]);
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                if (r == 1 && jb == jj) break;
                const long long o = (((long long)b * g.Ny + j0 + jj + r) * g.Nx + i) * 3;
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    if constexpr (sizeof(OUT) == 16)
                        out[o + c] = e[r][c];
                    else
                        out[o + c] = make_float2((float)e[r][c].x, (float)e[r][c].y);
                }
            }
        }
    }
}

template <int MAXM>
void launch_e_m(const FieldGeom& g, dim3 ge, cudaStream_t st, const double2* Ex, const double2* U, void* out,
                int precision) {
    if (precision == 0)
        field_e_kernel<double2, MAXM><<<ge, FE_THREADS, 0, st>>>(g, Ex, U, (double2*)out);
    else
        field_e_kernel<float2, MAXM><<<ge, FE_THREADS, 0, st>>>(g, Ex, U, (float2*)out);
}

sc_status launch_e(const FieldGeom& g, dim3 ge, cudaStream_t st, const double2* Ex, const double2* U, void* out,
                   int precision) {
    if (g.Mx <= 8) launch_e_m<8>(g, ge, st, Ex, U, out, precision);
    else if (g.Mx <= 16) launch_e_m<16>(g, ge, st, Ex, U, out, precision);
    else if (g.Mx <= 24) launch_e_m<24>(g, ge, st, Ex, U, out, precision);
    else if (g.Mx <= 32) launch_e_m<32>(g, ge, st, Ex, U, out, precision);
    else launch_e_m<FE_MAXM>(g, ge, st, Ex, U, out, precision);
    return SC_OK;
}

}  // namespace

sc_status volume_field_grid(sc_context* ctx, const sc_volume_params* p, int Z, int S1, int S2, const double2* x,
                            const double2* evl, const double2* Qc, const double2* Qh, int ez_mode,
                            const double* origin, const double* step, const int* counts, double zeps, void* out,
                            int precision, cudaStream_t st) {
    VolumePlan P;
    SC_TRY(make_plan(p, Z, S1, S2, &P));
    FieldGeom g;
    g.MF = P.dims.MF;
    g.Mx = P.dims.Mx;
    g.My = P.dims.My;
    g.Z = Z;
    g.external = p->external;
    g.Nx = counts[0];
    g.Ny = counts[1];
    g.Nz = counts[2];
    g.x0 = origin[0];
    g.y0 = origin[1];
    g.z0 = origin[2];
    g.dx = step[0];
    g.dy = step[1];
    g.dz = step[2];
    g.zeps = zeps;
    if (g.Nx <= 0 || g.Ny <= 0 || g.Nz <= 0 || g.Nz > 65535 / 3 || (precision != 0 && precision != 1)) {
        set_error("sc_volume_field_grid: bad grid or precision");
        return SC_BADINPUT;
    }
    if (g.Mx > FE_MAXM) {
        set_error("sc_volume_field_grid: %d orders along x exceed the grid evaluator's %d", g.Mx, FE_MAXM);
        return SC_BADINPUT;
    }
    if (!p->external && (!Qc || !Qh)) {
        set_error("sc_volume_field_grid: interior fields (Qc, Qh) missing");
        return SC_BADINPUT;
    }
    Workspace& ws = ctx->ws;
    const long long nw = 3LL * g.MF;   // compact table: Pi | Pr_0 | Pt_Z
    std::vector<double> hz(Z + 1);
    for (int l = 0; l <= Z; ++l) hz[l] = (p->external && l != 0 && l != Z) ? 0.0 : P.z[l];
    // planes of the interior regions (inside layer l = region - 1), grouped by layer, HQ_NPL per group
    std::vector<int> pidx;
    std::vector<PlaneGroup> groups;
    if (!p->external) {
        std::vector<std::vector<int>> by_layer(Z);
        for (int b = 0; b < g.Nz; ++b) {
            const double z = g.z0 + g.dz * b;
            int l = 0;
            for (int i = 0; i <= Z; ++i)
                if (z >= hz[i] - g.zeps) l = i + 1;
            if (l >= 1 && l <= Z) by_layer[l - 1].push_back(b);
        }
        for (int l = 0; l < Z; ++l)
            for (size_t q = 0; q < by_layer[l].size(); q += HQ_NPL) {
                const int cnt = (int)std::min<size_t>(HQ_NPL, by_layer[l].size() - q);
                groups.push_back(PlaneGroup{l, (int)pidx.size(), cnt});
                for (int r = 0; r < cnt; ++r) pidx.push_back(by_layer[l][q + r]);
            }
    }
    // device: compact wave table, boundary planes (as written to .cw), small arrays
    double2 *W, *svec, *Ex, *Ey, *H, *U, *Hp = nullptr;
    double *zpl, *zl, *kxy;
    PlaneGroup* dgroups = nullptr;
    int* dpidx = nullptr;
    SC_TRY(ws.get(&W, (size_t)nw * 6, WS_FIELD_W, st));
    SC_TRY(ws.get(&svec, (size_t)7 * g.MF, WS_EVAL_W, st));
    SC_TRY(ws.get(&zpl, (size_t)2 * (Z + 1) + g.Mx + g.My, WS_EVAL_IDX, st));
    zl = zpl + (Z + 1);
    kxy = zl + (Z + 1);
    if (!groups.empty()) {
        unsigned char* gbuf;
        const size_t gbytes = groups.size() * sizeof(PlaneGroup), ibytes = pidx.size() * sizeof(int);
        SC_TRY(ws.get(&gbuf, gbytes + ibytes + 16, WS_FIELD_G, st));
        dgroups = reinterpret_cast<PlaneGroup*>(gbuf);
        dpidx = reinterpret_cast<int*>(gbuf + ((gbytes + 15) / 16) * 16);
        SC_TRY(ws.get(&Hp, (size_t)HQ_JS * g.Nz * 3 * g.MF, WS_FIELD_HP, st));
    }
    SC_TRY(ws.get(&Ex, (size_t)g.Nx * g.Mx + (size_t)g.My * g.Ny, WS_FIELD_T, st));
    Ey = Ex + (size_t)g.Nx * g.Mx;
    SC_TRY(ws.get(&H, (size_t)g.Nz * 3 * g.MF, WS_FIELD_H, st));
    SC_TRY(ws.get(&U, (size_t)g.Nz * 3 * g.Mx * g.Ny, WS_FIELD_U, st));
    std::vector<cplx> hv;
    hv.insert(hv.end(), P.Sx.begin(), P.Sx.end());
    hv.insert(hv.end(), P.Sy.begin(), P.Sy.end());
    hv.insert(hv.end(), P.Sz0.begin(), P.Sz0.end());
    hv.insert(hv.end(), P.Sz1.begin(), P.Sz1.end());
    hv.insert(hv.end(), P.EF.begin(), P.EF.end());
    SC_CUDA_TRY(cudaMemcpyAsync(svec, hv.data(), hv.size() * sizeof(cplx), cudaMemcpyHostToDevice, st));
    SC_CUDA_TRY(cudaMemcpyAsync(zpl, P.z.data(), sizeof(double) * (Z + 1), cudaMemcpyHostToDevice, st));
    SC_CUDA_TRY(cudaMemcpyAsync(zl, hz.data(), sizeof(double) * (Z + 1), cudaMemcpyHostToDevice, st));
    if (!groups.empty()) {
        SC_CUDA_TRY(cudaMemcpyAsync(dgroups, groups.data(), sizeof(PlaneGroup) * groups.size(),
                                    cudaMemcpyHostToDevice, st));
        SC_CUDA_TRY(cudaMemcpyAsync(dpidx, pidx.data(), sizeof(int) * pidx.size(), cudaMemcpyHostToDevice, st));
    }
    for (int i = 0; i < 6; ++i)
        if (!ctx->ev[i]) SC_CUDA_TRY(cudaEventCreate(&ctx->ev[i]));
    SC_CUDA_TRY(cudaEventRecord(ctx->ev[0], st));
    double2* E0 = W;
    double2* K = W + (size_t)nw * 3;
    SC_TRY(volume_boundary_waves_launch(st, g.MF, Z, svec, x, zpl, P.dims.k, p->n[0], p->n[1], p->external, ez_mode,
                                        E0, K));
    double* kx = kxy;
    double* ky = kxy + g.Mx;
    field_k_kernel<<<(std::max(g.Mx, g.My) + 127) / 128, 128, 0, st>>>(g, K, kx, ky);
    const long long ntab = (long long)g.Nx * g.Mx + (long long)g.My * g.Ny;
    field_tables_kernel<<<(unsigned)((ntab + 255) / 256), 256, 0, st>>>(g, kx, ky, Ex, Ey);
    SC_CUDA_TRY(cudaEventRecord(ctx->ev[1], st));
    field_h_kernel<<<dim3(g.MF, g.Nz), FH_THREADS, 0, st>>>(g, E0, K, zl, H);
    if (!groups.empty()) {
        if (groups.size() > 65535) {
            set_error("sc_volume_field_grid: too many interior planes");
            return SC_BADINPUT;
        }
        field_hq_kernel<<<dim3((g.MF + HQ_P - 1) / HQ_P, (unsigned)groups.size(), HQ_JS), HQ_W * 32, 0, st>>>(
            g, P.dims.k, svec, svec + g.MF, evl, Qc, Qh, zpl, dgroups, dpidx, ez_mode, Hp);
        const long long tot = (long long)pidx.size() * 3 * g.MF;
        field_hq_sum_kernel<<<(unsigned)std::min<long long>((tot + 255) / 256, 65535), 256, 0, st>>>(
            g, dpidx, (int)pidx.size(), Hp, H);
        count_launch(2);
    }
    SC_CUDA_TRY(cudaEventRecord(ctx->ev[2], st));
    const long long per = (long long)g.Mx * g.Ny;
    field_u_kernel<<<dim3((unsigned)((per + 255) / 256), g.Nz * 3), 256, 0, st>>>(g, H, Ey, U);
    SC_CUDA_TRY(cudaEventRecord(ctx->ev[3], st));
    // y split so that the grid holds about eight CTAs per SM
    const int xblocks = (g.Nx + FE_THREADS - 1) / FE_THREADS;
    const int chunks = (g.Ny + FE_YCHUNK - 1) / FE_YCHUNK;
    int ysplit = (int)std::min<long long>(chunks, std::max<long long>(1, (148LL * 8) / ((long long)xblocks * g.Nz)));
    if (ysplit > 65535) ysplit = 65535;
    const dim3 ge(xblocks, g.Nz, ysplit);
    SC_TRY(launch_e(g, ge, st, Ex, U, out, precision));
    SC_CUDA_TRY(cudaEventRecord(ctx->ev[4], st));
    count_launch(5);
    SC_CHECK_LAUNCH("field grid");
    // stage times: wave table + tables, order sums, y transform, x transform
    SC_CUDA_TRY(cudaStreamSynchronize(st));
    for (double& v : ctx->stage_ms) v = 0.0;
    for (int i = 0; i < 4; ++i) {
        float ms = 0.f;
        SC_CUDA_TRY(cudaEventElapsedTime(&ms, ctx->ev[i], ctx->ev[i + 1]));
        ctx->stage_ms[i] = ms;
    }
    float tot = 0.f;
    SC_CUDA_TRY(cudaEventElapsedTime(&tot, ctx->ev[0], ctx->ev[4]));
    ctx->stage_ms[7] = tot;
    return SC_OK;
}

}  // namespace sc
