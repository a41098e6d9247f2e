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

sc_status volume_waves_launch(cudaStream_t st, int MF, int Z, const double2* svec, const double2* x,
                              const double2* evl, const double2* Qc, const double2* Qh, const double* zpl,
                              double k, double ntop, double nbot, int external, int ez_mode, long long nw,
                              double2* E0, double2* K);
void volume_regions(int MF, int Z, int external, long long* nw, int* begin, int* end);

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
                                                             const int* __restrict__ begin,
                                                             double2* __restrict__ H) {
    __shared__ double2 red[3][FH_THREADS];
    const int p = blockIdx.x, b = blockIdx.y;
    const int MF = g.MF;
    const double z = g.z0 + g.dz * b;
    int l = 0;
    for (int i = 0; i <= g.Z; ++i)
        if (z >= zl[i] - g.zeps) l = i + 1;
    // lists of region l: (start, waves per order)
    long long s0 = begin[l], s1 = -1;
    long long m0 = 1, m1 = 1;
    const long long internal = (long long)2 * MF * MF;
    if (l == 0) {
        s1 = s0 + MF;                      // Pi, then Pr_0
    } else if (l <= g.Z) {
        if (g.external) s0 = -1;           // no internal waves
        else {
            m0 = m1 = 2LL * MF;             // Pt_{l-1}, then Pr_l
            s1 = s0 + internal;
        }
    }                                      // l == Z + 1: Pt_Z alone
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
        for (int jj = 0; jj < nj; ++jj) {
            double2 e[3] = {make_double2(0.0, 0.0), make_double2(0.0, 0.0), make_double2(0.0, 0.0)};
#pragma unroll
            for (int px = 0; px < MAXM; ++px) {
                if (px < Mx) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) e[c] = cfma(ex[px], su[jj][c][px], e[c]);
                }
            }
            const long long o = (((long long)b * g.Ny + j0 + jj) * g.Nx + i) * 3;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                if constexpr (sizeof(OUT) == 16)
                    out[o + c] = e[c];
                else
                    out[o + c] = make_float2((float)e[c].x, (float)e[c].y);
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
    long long nw = 0;
    std::vector<int> hb(Z + 2), he(Z + 2);
    volume_regions(g.MF, Z, p->external, &nw, hb.data(), he.data());
    std::vector<double> hz(Z + 1);
    for (int l = 0; l <= Z; ++l) hz[l] = (p->external && l != 0 && l != Z) ? 0.0 : P.z[l];
    // device: wave table, region starts, boundary planes (as written to .cw), small arrays
    double2 *W, *svec, *Ex, *Ey, *H, *U;
    double *zpl, *zl, *kxy;
    int* dbeg;
    SC_TRY(ws.get(&W, (size_t)nw * 6, WS_FIELD_W, st));
    SC_TRY(ws.get(&svec, (size_t)7 * g.MF, WS_EVAL_W, st));
    SC_TRY(ws.get(&zpl, (size_t)2 * (Z + 1) + g.Mx + g.My, WS_EVAL_IDX, st));
    zl = zpl + (Z + 1);
    kxy = zl + (Z + 1);
    SC_TRY(ws.get(&dbeg, (size_t)Z + 2, WS_BINS, st));
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
    SC_CUDA_TRY(cudaMemcpyAsync(dbeg, hb.data(), sizeof(int) * (Z + 2), cudaMemcpyHostToDevice, st));
    for (int i = 0; i < 6; ++i)
        if (!ctx->ev[i]) SC_CUDA_TRY(cudaEventCreate(&ctx->ev[i]));
    SC_CUDA_TRY(cudaEventRecord(ctx->ev[0], st));
    double2* E0 = W;
    double2* K = W + (size_t)nw * 3;
    SC_TRY(volume_waves_launch(st, g.MF, Z, svec, x, evl, Qc, Qh, zpl, P.dims.k, p->n[0], p->n[1], p->external,
                               ez_mode, nw, E0, K));
    double* kx = kxy;
    double* ky = kxy + g.Mx;
    field_k_kernel<<<(std::max(g.Mx, g.My) + 127) / 128, 128, 0, st>>>(g, K, kx, ky);
    const long long ntab = (long long)g.Nx * g.Mx + (long long)g.My * g.Ny;
    field_tables_kernel<<<(unsigned)((ntab + 255) / 256), 256, 0, st>>>(g, kx, ky, Ex, Ey);
    SC_CUDA_TRY(cudaEventRecord(ctx->ev[1], st));
    field_h_kernel<<<dim3(g.MF, g.Nz), FH_THREADS, 0, st>>>(g, E0, K, zl, dbeg, H);
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
