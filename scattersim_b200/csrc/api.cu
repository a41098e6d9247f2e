// extern "C" entry points of libscattersim_b200 (declared in
// include/scattersim_b200.h).  Every function validates its arguments, maps
// CUDA failures to SC_CUDA_ERROR and records a message for
// sc_last_error_string(); nothing exits or traps.
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "context.cuh"

namespace sc {

static thread_local char g_err[512] = "";
static std::atomic<uint64_t> g_launches{0};

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

sc_status cuda_status(cudaError_t e, const char* where) {
    set_error("%s: %s", where, cudaGetErrorString(e));
    if (e == cudaErrorMemoryAllocation) return SC_OOM;
    return SC_CUDA_ERROR;
}

void count_launch(int n) { g_launches.fetch_add((uint64_t)n, std::memory_order_relaxed); }
uint64_t launch_total() { return g_launches.load(); }

sc_status smem_opt_in(const void* kernel, int bytes) {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, int> granted;   // (kernel, device) -> bytes
    int dev = 0;
    SC_CUDA_TRY(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lock(mu);
    int& have = granted[{kernel, dev}];
    if (have >= bytes) return SC_OK;
    SC_CUDA_TRY(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    have = bytes;
    return SC_OK;
}

sc_status set_volume_precision(sc_context* ctx, int precision);
sc_status sweep_solve(sc_context* ctx, int count, const sc_volume_params* params, const void* const* samples,
                      const int* Zs, const int* S1s, const int* S2s, void* const* x_out, int precision,
                      int* status, cudaStream_t st);
sc_status volume_solve(sc_context* ctx, const sc_volume_params* p, const double2* sample, int Z, int S1,
                       int S2, double2* x_out, double2* evl_out, double2* Qc_out, double2* Qh_out,
                       int* info_host, cudaStream_t st);
sc_status volume_chain_block(sc_context* ctx, const sc_volume_params* p, const double2* sample, int Z, int S1,
                             int S2, int lb, int le, double2* P_out, double2* GD0_out, int* info_host,
                             cudaStream_t st);
sc_status volume_boundary_solve(sc_context* ctx, const sc_volume_params* p, int Z, int S1, int S2,
                                const double2* Gcs_in, const double2* GD0, double2* x_out, int* info_host,
                                cudaStream_t st);
sc_status volume_field_grid(sc_context* ctx, const sc_volume_params* p, int Z, int S1, int S2, const double2* x,
                            const double2* evl, const double2* Qc, const double2* Qh, int ez_mode,
                            const double* origin, const double* step, const int* counts, double zeps, void* out,
                            int precision, cudaStream_t st);
sc_status cw_write(sc_context* ctx, const char* path, const double2* E0, const double2* K, long long nw, int layers,
                   const double* z_layers, const long long* counts, int frame, cudaStream_t st);
sc_status volume_waves_launch(cudaStream_t st, int MF, int Z, const double2* svec, const double2* x,
                              const double2* evl, const double2* Qc, const double2* Qh, const double* zpl,
                              double k, double ntop, double nbot, int external, int ez_mode, long long nw,
                              double2* E0, double2* K);
sc_status cw_evaluate_launch(cudaStream_t st, const double2* E0, const double2* K, const double* zl,
                             const int* begin, const int* end, int layers, double zeps, const double* pts,
                             long long np, double2* out, int precision);

namespace {
struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        cudaGetDevice(&prev);
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        cudaGetDevice(&cur);
        if (prev >= 0 && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace

// region index of a scattervolume wave table (cw_allocate, cpuEvaluator.cpp:34-53)
void volume_regions(int MF, int Z, int external, long long* nw, int* begin, int* end) {
    const long long internal = 2LL * MF * MF;
    long long total = MF;
    begin[0] = 0;
    for (int l = 0; l <= Z; ++l) {
        long long npr = (l == 0) ? MF : (external ? 0 : internal);
        long long npt = (l == Z) ? MF : (external ? 0 : internal);
        total += npr;
        end[l] = (int)total;
        begin[l + 1] = (int)total;
        total += npt;
    }
    end[Z + 1] = (int)total;
    *nw = total;
}

}  // namespace sc

using namespace sc;

extern "C" {

const char* sc_version(void) { return "scattersim_b200 0.1 (sm_100a)"; }

const char* sc_last_error_string(void) { return g_err; }

sc_status sc_create(sc_context** ctx, int device) {
    if (!ctx) {
        set_error("sc_create: null ctx");
        return SC_BADINPUT;
    }
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess) return cuda_status(e, "cudaGetDeviceCount");
    if (device < 0 || device >= count) {
        set_error("sc_create: device %d out of range (%d devices)", device, count);
        return SC_BADINPUT;
    }
    DeviceGuard g(device);
    cudaFree(nullptr);
    auto* c = new sc_context();
    c->device = device;
    c->launches_at_create = launch_total();
    *ctx = c;
    return SC_OK;
}

sc_status sc_destroy(sc_context* ctx) {
    if (!ctx) return SC_OK;
    DeviceGuard g(ctx->device);
    cudaDeviceSynchronize();
    ctx->ws.release();
    for (auto& ev : ctx->ev)
        if (ev) cudaEventDestroy(ev);
    delete ctx;
    return SC_OK;
}

uint64_t sc_launch_count(const sc_context* ctx) {
    (void)ctx;
    return launch_total();
}

sc_status sc_fft2_crop(sc_context* ctx, const void* sample, int Z, int S1, int S2, int Mx, int My, void* Nf,
                       void* Nif, void* stream) {
    if (!ctx || !sample || !Nf || !Nif) {
        set_error("sc_fft2_crop: null argument");
        return SC_BADINPUT;
    }
    DeviceGuard g(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    double2 *R2, *Ri2;
    int* bins;
    SC_TRY(ctx->ws.get(&R2, (size_t)Z * S1 * Mx, WS_TMP, st));
    SC_TRY(ctx->ws.get(&Ri2, (size_t)Z * S1 * Mx, WS_TMP2, st));
    SC_TRY(ctx->ws.get(&bins, (size_t)Mx + My, WS_BINS, st));
    SC_TRY(fft2_crop(st, (const double2*)sample, Z, S1, S2, Mx, My, (double2*)Nf, (double2*)Nif, R2, Ri2, bins));
    SC_CUDA_TRY(cudaStreamSynchronize(st));
    return SC_OK;
}

sc_status sc_phi(sc_context* ctx, const void* Nf, const void* Nif, int Z, int Mx, int My, const double* up_host,
                 const double* wq_host, double k, void* Phi, void* stream) {
    if (!ctx || !Nf || !Nif || !up_host || !wq_host || !Phi || Z <= 0 || Mx <= 0 || My <= 0) {
        set_error("sc_phi: bad argument");
        return SC_BADINPUT;
    }
    DeviceGuard g(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    double* lat;
    SC_TRY(ctx->ws.get(&lat, (size_t)Mx + My, WS_LAT, st));
    std::vector<double> h(up_host, up_host + Mx);
    h.insert(h.end(), wq_host, wq_host + My);
    SC_CUDA_TRY(cudaMemcpyAsync(lat, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, st));
    SC_TRY(assemble_phi(st, (const double2*)Nf, (const double2*)Nif, Z, Mx, My, lat, k, (double2*)Phi));
    SC_CUDA_TRY(cudaStreamSynchronize(st));
    return SC_OK;
}

sc_status sc_eigensolve_batched(sc_context* ctx, void* A, int n, int batch, void* evl, void* evt, int* info,
                                void* stream) {
    if (!ctx || !A || !evl || !evt || n <= 0 || batch <= 0) {
        set_error("sc_eigensolve_batched: bad argument");
        return SC_BADINPUT;
    }
    DeviceGuard g(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    int* dinfo;
    SC_TRY(ctx->ws.get(&dinfo, (size_t)batch, WS_INFO, st));
    SC_CUDA_TRY(cudaMemsetAsync(dinfo, 0, sizeof(int) * batch, st));
    SC_TRY(eig_batched(st, (double2*)A, n, batch, (double2*)evl, (double2*)evt, dinfo, ctx->ws));
    std::vector<int> h(batch);
    SC_CUDA_TRY(cudaMemcpyAsync(h.data(), dinfo, sizeof(int) * batch, cudaMemcpyDeviceToHost, st));
    SC_CUDA_TRY(cudaStreamSynchronize(st));
    int bad = 0;
    for (int b = 0; b < batch; ++b) {
        if (info) info[b] = h[b];
        if (h[b]) bad = 1;
    }
    if (bad) {
        set_error("sc_eigensolve_batched: QR iteration cap reached");
        return SC_NOCONVERGE;
    }
    return SC_OK;
}

sc_status sc_linearsolve_batched(sc_context* ctx, void* A, int n, void* B, int nrhs, int batch, int* info,
                                 void* stream) {
    if (!ctx || !A || !B || n <= 0 || nrhs <= 0 || batch <= 0) {
        set_error("sc_linearsolve_batched: bad argument");
        return SC_BADINPUT;
    }
    DeviceGuard g(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    int *piv, *dinfo;
    SC_TRY(ctx->ws.get(&piv, (size_t)batch * n, WS_PIV, st));
    SC_TRY(ctx->ws.get(&dinfo, (size_t)batch, WS_INFO, st));
    SC_CUDA_TRY(cudaMemsetAsync(dinfo, 0, sizeof(int) * batch, st));
    const long long sA = (long long)n * n, sB = (long long)n * nrhs;
    SC_TRY(getrf(st, (double2*)A, n, sA, n, batch, piv, dinfo));
    SC_TRY(getrs(st, (const double2*)A, n, sA, n, piv, (double2*)B, n, sB, nrhs, batch));
    std::vector<int> h(batch);
    SC_CUDA_TRY(cudaMemcpyAsync(h.data(), dinfo, sizeof(int) * batch, cudaMemcpyDeviceToHost, st));
    SC_CUDA_TRY(cudaStreamSynchronize(st));
    int bad = 0;
    for (int b = 0; b < batch; ++b) {
        if (info) info[b] = h[b];
        if (h[b]) bad = 1;
    }
    if (bad) {
        set_error("sc_linearsolve_batched: exactly singular matrix");
        return SC_SINGULAR;
    }
    return SC_OK;
}

sc_status sc_inverse_batched(sc_context* ctx, const void* A, int n, int batch, void* Ainv, int* info,
                             void* stream) {
    if (!ctx || !A || !Ainv || n <= 0 || batch <= 0) {
        set_error("sc_inverse_batched: bad argument");
        return SC_BADINPUT;
    }
    DeviceGuard g(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    const long long sA = (long long)n * n;
    double2* LU;
    SC_TRY(ctx->ws.get(&LU, (size_t)batch * sA, WS_GD, st));
    SC_CUDA_TRY(cudaMemcpyAsync(LU, A, sizeof(double2) * batch * sA, cudaMemcpyDeviceToDevice, st));
    SC_TRY(set_identity(st, (double2*)Ainv, n, sA, n, batch));
    return sc_linearsolve_batched(ctx, LU, n, Ainv, n, batch, info, stream);
}

namespace {
// the int8 tensor-core engines behind one C entry each: slices 1..7 = digit
// slices, 0 = modular (CRT)
sc_status int8_gemm_entry(const char* name, sc_context* ctx, int slices, int m, int n, int k, const double* alpha,
                          const void* A, int lda, long long strideA, const void* B, int ldb, long long strideB,
                          const double* beta, void* C, int ldc, long long strideC, int batch, void* stream) {
    if (!ctx || !alpha || !beta || !A || !B || !C || m < 0 || n < 0 || k < 0 || batch < 0 ||
        lda < (m > 1 ? m : 1) || ldb < (k > 1 ? k : 1) || ldc < (m > 1 ? m : 1)) {
        set_error("%s: bad argument", name);
        return SC_BADINPUT;
    }
    DeviceGuard g(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    int* err;
    SC_TRY(ctx->ws.get(&err, 1, WS_OZ_ERR, st));
    SC_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), st));
    GemmArgs a;
    a.m = m;
    a.n = n;
    a.k = k;
    a.alpha = make_double2(alpha[0], alpha[1]);
    a.beta = make_double2(beta[0], beta[1]);
    a.A = (const double2*)A;
    a.lda = lda;
    a.sA = strideA;
    a.B = (const double2*)B;
    a.ldb = ldb;
    a.sB = strideB;
    a.C = (double2*)C;
    a.ldc = ldc;
    a.sC = strideC;
    if (slices > 0)
        SC_TRY(zgemm_ozaki(st, slices, a, batch, ctx->ws, err));
    else
        SC_TRY(zgemm_crt(st, a, batch, ctx->ws, err));
    int herr = 0;
    SC_CUDA_TRY(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    SC_CUDA_TRY(cudaStreamSynchronize(st));
    if (herr) {
        set_error("%s: tensor-core pipeline wait timed out (stage %d)", name, herr);
        return SC_CUDA_ERROR;
    }
    return SC_OK;
}
}  // namespace

sc_status sc_zgemm_emulated_batched(sc_context* ctx, int slices, int m, int n, int k, const double* alpha,
                                    const void* A, int lda, long long strideA, const void* B, int ldb,
                                    long long strideB, const double* beta, void* C, int ldc, long long strideC,
                                    int batch, void* stream) {
    if (slices < 1 || slices > 7) {
        set_error("sc_zgemm_emulated_batched: slices must be 1..7");
        return SC_BADINPUT;
    }
    return int8_gemm_entry("sc_zgemm_emulated_batched", ctx, slices, m, n, k, alpha, A, lda, strideA, B, ldb,
                           strideB, beta, C, ldc, strideC, batch, stream);
}

sc_status sc_zgemm_crt_batched(sc_context* ctx, int m, int n, int k, const double* alpha, const void* A, int lda,
                               long long strideA, const void* B, int ldb, long long strideB, const double* beta,
                               void* C, int ldc, long long strideC, int batch, void* stream) {
    return int8_gemm_entry("sc_zgemm_crt_batched", ctx, 0, m, n, k, alpha, A, lda, strideA, B, ldb, strideB, beta, C,
                           ldc, strideC, batch, stream);
}

sc_status sc_zgemm_batched(sc_context* ctx, int m, int n, int k, const double* alpha, const void* A, int lda,
                           long long strideA, const void* B, int ldb, long long strideB, const double* beta,
                           void* C, int ldc, long long strideC, int batch, void* stream) {
    if (!ctx || !alpha || !beta || !A || !B || !C || m < 0 || n < 0 || k < 0 || lda < (m > 1 ? m : 1) ||
        ldb < (k > 1 ? k : 1) || ldc < (m > 1 ? m : 1)) {
        set_error("sc_zgemm_batched: bad argument");
        return SC_BADINPUT;
    }
    DeviceGuard g(ctx->device);
    return zgemm((cudaStream_t)stream, m, n, k, make_double2(alpha[0], alpha[1]), (const double2*)A, lda, strideA,
                 (const double2*)B, ldb, strideB, make_double2(beta[0], beta[1]), (double2*)C, ldc, strideC,
                 batch);
}

void sc_volume_params_default(sc_volume_params* p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->lambda = 1.0;
    p->direction[2] = 1.0;
    p->ey[0] = 1.0;
    p->n[0] = p->n[1] = 1.0;
    p->size[0] = 10.0;
    p->size[1] = 10.0;
    p->size[2] = 2.0;
}

sc_status sc_volume_plan(const sc_volume_params* p, int Z, int S1, int S2, sc_volume_dims* dims) {
    if (!dims) {
        set_error("sc_volume_plan: null dims");
        return SC_BADINPUT;
    }
    VolumePlan P;
    SC_TRY(make_plan(p, Z, S1, S2, &P));
    *dims = P.dims;
    return SC_OK;
}

sc_status sc_volume_solve(sc_context* ctx, const sc_volume_params* p, const void* sample, int Z, int S1, int S2,
                          void* x, void* evl, void* Qc, void* Qh, int* info, void* stream) {
    if (!ctx || !p || !sample) {
        set_error("sc_volume_solve: null argument");
        return SC_BADINPUT;
    }
    DeviceGuard g(ctx->device);
    return volume_solve(ctx, p, (const double2*)sample, Z, S1, S2, (double2*)x, (double2*)evl, (double2*)Qc,
                        (double2*)Qh, info, (cudaStream_t)stream);
}

sc_status sc_volume_chain_block(sc_context* ctx, const sc_volume_params* p, const void* sample, int Z, int S1,
                                int S2, int layer_begin, int layer_end, void* P, void* GD0, int* info, void* stream) {
    if (!ctx || !p || !sample || !P) {
        set_error("sc_volume_chain_block: null argument");
        return SC_BADINPUT;
    }
    DeviceGuard g(ctx->device);
    return volume_chain_block(ctx, p, (const double2*)sample, Z, S1, S2, layer_begin, layer_end, (double2*)P,
                              (double2*)GD0, info, (cudaStream_t)stream);
}

sc_status sc_volume_boundary_solve(sc_context* ctx, const sc_volume_params* p, int Z, int S1, int S2,
                                   const void* Gc_static, const void* GD0, void* x, int* info, void* stream) {
    if (!ctx || !p || !Gc_static || !GD0 || !x) {
        set_error("sc_volume_boundary_solve: null argument");
        return SC_BADINPUT;
    }
    DeviceGuard g(ctx->device);
    return volume_boundary_solve(ctx, p, Z, S1, S2, (const double2*)Gc_static, (const double2*)GD0, (double2*)x,
                                 info, (cudaStream_t)stream);
}

sc_status sc_sweep_solve(sc_context* ctx, int count, const sc_volume_params* params, const void* const* samples,
                         const int* Z, const int* S1, const int* S2, void* const* x, int precision, int* status,
                         void* stream) {
    if (!ctx) {
        set_error("sc_sweep_solve: null context");
        return SC_BADINPUT;
    }
    DeviceGuard g(ctx->device);
    return sweep_solve(ctx, count, params, samples, Z, S1, S2, x, precision, status, (cudaStream_t)stream);
}

sc_status sc_kernel_timing(sc_context* ctx, int on) {
    if (!ctx) {
        set_error("sc_kernel_timing: null context");
        return SC_BADINPUT;
    }
    DeviceGuard g(ctx->device);
    Workspace& ws = ctx->ws;
    SC_CUDA_TRY(cudaDeviceSynchronize());
    for (auto& m : ws.marks) {
        ws.event_pool.push_back(m.e0);
        ws.event_pool.push_back(m.e1);
    }
    ws.marks.clear();
    ws.time_kernels = on != 0;
    return SC_OK;
}

sc_status sc_kernel_stats(sc_context* ctx, double* out8) {
    if (!ctx || !out8) {
        set_error("sc_kernel_stats: null argument");
        return SC_BADINPUT;
    }
    DeviceGuard g(ctx->device);
    SC_CUDA_TRY(cudaDeviceSynchronize());
    for (int i = 0; i < 8; ++i) out8[i] = 0.0;
    for (auto& m : ctx->ws.marks) {
        if (m.cls > 1) continue;
        float ms = 0.f;
        SC_CUDA_TRY(cudaEventElapsedTime(&ms, m.e0, m.e1));
        double* o = out8 + 4 * m.cls;
        o[0] += 1.0;
        o[1] += ms;
        o[2] += m.flops;
        o[3] += m.int8_ops;
    }
    return SC_OK;
}

sc_status sc_kernel_stats_ex(sc_context* ctx, double* out, int classes) {
    if (!ctx || !out || classes < 0) {
        set_error("sc_kernel_stats_ex: bad argument");
        return SC_BADINPUT;
    }
    DeviceGuard g(ctx->device);
    SC_CUDA_TRY(cudaDeviceSynchronize());
    for (int i = 0; i < 4 * classes; ++i) out[i] = 0.0;
    for (auto& m : ctx->ws.marks) {
        if (m.cls >= classes) continue;
        float ms = 0.f;
        SC_CUDA_TRY(cudaEventElapsedTime(&ms, m.e0, m.e1));
        double* o = out + 4 * m.cls;
        o[0] += 1.0;
        o[1] += ms;
        o[2] += m.flops;
        o[3] += m.int8_ops;
    }
    return SC_OK;
}

sc_status sc_gemm_choices_get(sc_context* ctx, int* rec, int cap, int* count) {
    if (!ctx || !count || (cap > 0 && !rec)) {
        set_error("sc_gemm_choices_get: null argument");
        return SC_BADINPUT;
    }
    int i = 0;
    for (auto& kv : ctx->ws.gemm_choice) {
        if (i < cap) {
            int* r = rec + 6 * i;
            r[0] = std::get<0>(kv.first);
            r[1] = std::get<1>(kv.first);
            r[2] = std::get<2>(kv.first);
            r[3] = std::get<3>(kv.first);
            r[4] = std::get<4>(kv.first);
            r[5] = kv.second;
        }
        ++i;
    }
    *count = i;
    return SC_OK;
}

sc_status sc_gemm_choices_set(sc_context* ctx, const int* rec, int count) {
    if (!ctx || count < 0 || (count > 0 && !rec)) {
        set_error("sc_gemm_choices_set: bad argument");
        return SC_BADINPUT;
    }
    for (int i = 0; i < count; ++i)
        if (rec[6 * i + 5] < 0 || rec[6 * i + 5] > 3) {
            set_error("sc_gemm_choices_set: record %d has unknown variant %d", i, rec[6 * i + 5]);
            return SC_BADINPUT;
        }
    ctx->ws.gemm_choice.clear();
    for (int i = 0; i < count; ++i) {
        const int* r = rec + 6 * i;
        ctx->ws.gemm_choice[std::make_tuple(r[0], r[1], r[2], r[3], r[4])] = r[5];
    }
    return SC_OK;
}

sc_status sc_volume_precision(sc_context* ctx, int precision) {
    if (!ctx) {
        set_error("sc_volume_precision: null context");
        return SC_BADINPUT;
    }
    return set_volume_precision(ctx, precision);
}

sc_status sc_volume_stage_ms(const sc_context* ctx, double* ms8) {
    if (!ctx || !ms8) {
        set_error("sc_volume_stage_ms: null argument");
        return SC_BADINPUT;
    }
    for (int i = 0; i < 8; ++i) ms8[i] = ctx->stage_ms[i];
    return SC_OK;
}

}  // extern "C"

namespace sc {
namespace probe {
// FP64 pipe probes: 8 independent DFMA chains per thread, or 4 independent
// DMMA m8n8k4 accumulators per warp; both sized to keep every SM's FP64 pipe busy
__global__ void fp64_dfma_kernel(double* out, int iters) {
    double a[8];
    for (int i = 0; i < 8; ++i) a[i] = threadIdx.x * 1e-9 + i;
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int u = 0; u < 16; ++u)
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = fma(a[i], 0.999999, 1e-7);
    double s = 0;
    for (int i = 0; i < 8; ++i) s += a[i];
    if (s == 1.2345) out[0] = s;
}
__global__ void fp64_dmma_kernel(double* out, int iters) {
    const double a = threadIdx.x * 1e-9, b = 1.0;
    double c[4][2];
    for (int i = 0; i < 4; ++i) c[i][0] = c[i][1] = 0.0;
    for (int it = 0; it < iters; ++it)
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int i = 0; i < 4; ++i)
                asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                             : "+d"(c[i][0]), "+d"(c[i][1])
                             : "d"(a), "d"(b));
    double s = 0;
    for (int i = 0; i < 4; ++i) s += c[i][0] + c[i][1];
    if (s == 1.2345) out[0] = s;
}
}  // namespace probe

static sc_status fp64_probe(sc_context* ctx, bool dmma, double* tflops) {
    DeviceGuard g(ctx->device);
    int sms = 0;
    SC_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device));
    double* out;
    SC_TRY(ctx->ws.get(&out, 1, WS_TMP, 0));
    const int blocks = sms * 8, threads = 256, iters = 4096;
    cudaEvent_t e0, e1;
    SC_CUDA_TRY(cudaEventCreate(&e0));
    SC_CUDA_TRY(cudaEventCreate(&e1));
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(e0, 0);
        if (dmma)
            probe::fp64_dmma_kernel<<<blocks, threads>>>(out, iters);
        else
            probe::fp64_dfma_kernel<<<blocks, threads>>>(out, iters);
        count_launch();
        cudaEventRecord(e1, 0);
        SC_CUDA_TRY(cudaEventSynchronize(e1));
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const double warps = (double)blocks * threads / 32.0;
    const double flops = dmma ? warps * iters * 16 * 2.0 * 8 * 8 * 4 : 2.0 * 16 * 8 * (double)iters * blocks * threads;
    *tflops = flops / (best * 1e-3) / 1e12;
    return SC_OK;
}
}  // namespace sc

extern "C" {

sc_status sc_fp64_peak_probe(sc_context* ctx, double* tflops) {
    if (!ctx || !tflops) {
        set_error("sc_fp64_peak_probe: null argument");
        return SC_BADINPUT;
    }
    return fp64_probe(ctx, false, tflops);
}

sc_status sc_fp64_dmma_probe(sc_context* ctx, double* tflops) {
    if (!ctx || !tflops) {
        set_error("sc_fp64_dmma_probe: null argument");
        return SC_BADINPUT;
    }
    return fp64_probe(ctx, true, tflops);
}

sc_status sc_crt_tiles_set(sc_context* ctx, int mode) {
    if (!ctx || (mode != 0 && mode != 1)) {
        set_error(ctx ? "sc_crt_tiles_set: mode %d, must be 0 or 1" : "sc_crt_tiles_set: null context", mode);
        return SC_BADINPUT;
    }
    ctx->ws.crt_tiles = mode;
    return SC_OK;
}

sc_status sc_int8_peak_probe(sc_context* ctx, double* tops) {
    if (!ctx || !tops) {
        set_error("sc_int8_peak_probe: null argument");
        return SC_BADINPUT;
    }
    DeviceGuard g(ctx->device);
    return int8_peak_probe(ctx->device, ctx->ws, tops);
}

sc_status sc_qr_stats(sc_context* ctx, long long* out, int count) {
    if (!ctx || !out || count < 0) {
        set_error("sc_qr_stats: bad argument");
        return SC_BADINPUT;
    }
    DeviceGuard g(ctx->device);
    const int nb = count < ctx->ws.hqr_batch ? count : ctx->ws.hqr_batch;
    if (nb > 0 && ctx->ws.hqr_stats) {
        SC_CUDA_TRY(cudaDeviceSynchronize());
        SC_CUDA_TRY(cudaMemcpy(out, ctx->ws.hqr_stats, sizeof(long long) * 8 * nb, cudaMemcpyDeviceToHost));
    }
    for (long long i = (long long)nb * 8; i < (long long)count * 8; ++i) out[i] = 0;
    return SC_OK;
}

sc_status sc_volume_waves(sc_context* ctx, const sc_volume_params* p, int Z, int S1, int S2, const void* x,
                          const void* evl, const void* Qc, const void* Qh, int ez_mode, long long* nw, int* begin,
                          int* end, double* z_layers, void* E0, void* k, void* stream) {
    if (!ctx || !p || !nw) {
        set_error("sc_volume_waves: null argument");
        return SC_BADINPUT;
    }
    VolumePlan P;
    SC_TRY(make_plan(p, Z, S1, S2, &P));
    const int MF = P.dims.MF;
    std::vector<int> b(Z + 2), e(Z + 2);
    volume_regions(MF, Z, p->external, nw, b.data(), e.data());
    if (begin) std::memcpy(begin, b.data(), sizeof(int) * (Z + 2));
    if (end) std::memcpy(end, e.data(), sizeof(int) * (Z + 2));
    if (z_layers) {
        // the .cw keeps z = 0 for interior boundaries written with --external
        for (int l = 0; l <= Z; ++l)
            z_layers[l] = (p->external && l != 0 && l != Z) ? 0.0 : P.z[l];
    }
    if (!E0 || !k) return SC_OK;
    if (!x || !evl || (!p->external && (!Qc || !Qh))) {
        set_error("sc_volume_waves: solution buffers missing");
        return SC_BADINPUT;
    }
    DeviceGuard g(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    double2* svec;
    double* zpl;
    SC_TRY(ctx->ws.get(&svec, (size_t)7 * MF, WS_EVAL_W, st));
    SC_TRY(ctx->ws.get(&zpl, (size_t)Z + 1, WS_EVAL_IDX, st));
    std::vector<cplx> hv;
    hv.insert(hv.end(), P.Sx.begin(), P.Sx.end());
    hv.insert(hv.end(), P.Sy.begin(), P.Sy.end());
    hv.insert(hv.end(), P.Sz0.begin(), P.Sz0.end());
    hv.insert(hv.end(), P.Sz1.begin(), P.Sz1.end());
    hv.insert(hv.end(), P.EF.begin(), P.EF.end());
    SC_CUDA_TRY(cudaMemcpyAsync(svec, hv.data(), hv.size() * sizeof(cplx), cudaMemcpyHostToDevice, st));
    SC_CUDA_TRY(cudaMemcpyAsync(zpl, P.z.data(), sizeof(double) * (Z + 1), cudaMemcpyHostToDevice, st));
    SC_TRY(volume_waves_launch(st, MF, Z, svec, (const double2*)x, (const double2*)evl, (const double2*)Qc,
                               (const double2*)Qh, zpl, P.dims.k, p->n[0], p->n[1], p->external, ez_mode, *nw,
                               (double2*)E0, (double2*)k));
    SC_CUDA_TRY(cudaStreamSynchronize(st));
    return SC_OK;
}

sc_status sc_volume_field_grid(sc_context* ctx, const sc_volume_params* p, int Z, int S1, int S2, const void* x,
                               const void* evl, const void* Qc, const void* Qh, int ez_mode, const double* origin,
                               const double* step, const int* counts, double zeps, void* out, int precision,
                               void* stream) {
    if (!ctx || !p || !x || !evl || !origin || !step || !counts || !out) {
        set_error("sc_volume_field_grid: null argument");
        return SC_BADINPUT;
    }
    DeviceGuard g(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    SC_TRY(volume_field_grid(ctx, p, Z, S1, S2, (const double2*)x, (const double2*)evl, (const double2*)Qc,
                             (const double2*)Qh, ez_mode, origin, step, counts, zeps, out, precision, st));
    return SC_OK;
}

sc_status sc_cw_write(sc_context* ctx, const char* path, const void* E0, const void* k, long long nw, int layers,
                      const double* z_layers, const long long* counts, int frame, void* stream) {
    if (!ctx || !path || layers < 0 || nw < 0 || !counts || (layers > 0 && !z_layers) || (nw > 0 && (!E0 || !k)) ||
        frame < 0 || frame > 2) {
        set_error("sc_cw_write: bad argument");
        return SC_BADINPUT;
    }
    DeviceGuard g(ctx->device);
    return cw_write(ctx, path, (const double2*)E0, (const double2*)k, nw, layers, z_layers, counts, frame,
                    (cudaStream_t)stream);
}

sc_status sc_cw_evaluate(sc_context* ctx, const void* E0, const void* k, int nw, const double* z_layers,
                         const int* begin, const int* end, int layers, double zeps, const double* points,
                         long long np, void* out, int precision, void* stream) {
    if (!ctx || !z_layers || !begin || !end || !points || !out || layers < 0 || nw < 0 ||
        (nw > 0 && (!E0 || !k)) || (precision != 0 && precision != 1)) {
        set_error("sc_cw_evaluate: bad argument");
        return SC_BADINPUT;
    }
    for (int l = 0; l <= layers; ++l) {
        if (begin[l] < 0 || end[l] < begin[l] || end[l] > nw) {
            set_error("sc_cw_evaluate: region %d [%d, %d) outside the %d waves", l, begin[l], end[l], nw);
            return SC_BADINPUT;
        }
    }
    DeviceGuard g(ctx->device);
    cudaStream_t st = (cudaStream_t)stream;
    int* idx;
    double* zl;
    SC_TRY(ctx->ws.get(&idx, (size_t)2 * (layers + 1), WS_EVAL_IDX, st));
    SC_TRY(ctx->ws.get(&zl, (size_t)layers + 1, WS_LAT, st));
    std::vector<int> hidx(begin, begin + layers + 1);
    hidx.insert(hidx.end(), end, end + layers + 1);
    SC_CUDA_TRY(cudaMemcpyAsync(idx, hidx.data(), sizeof(int) * hidx.size(), cudaMemcpyHostToDevice, st));
    if (layers > 0)
        SC_CUDA_TRY(cudaMemcpyAsync(zl, z_layers, sizeof(double) * layers, cudaMemcpyHostToDevice, st));
    SC_TRY(cw_evaluate_launch(st, (const double2*)E0, (const double2*)k, zl, idx, idx + layers + 1, layers, zeps,
                              points, np, (double2*)out, precision));
    SC_CUDA_TRY(cudaStreamSynchronize(st));
    return SC_OK;
}

// ------------------------------------------------- layers and focused beams
sc_status sc_beam_polar(sc_context* ctx, double alpha, double beta, int N0, int N1, const double* k_center,
                        const double* E_center, const double* focus, double* k_out, void* E_out, int* count,
                        void* stream) {
    if (!ctx) {
        set_error("sc_beam_polar: null context");
        return SC_BADINPUT;
    }
    DeviceGuard g(ctx->device);
    return beam_polar((cudaStream_t)stream, alpha, beta, N0, N1, k_center, (const double2*)E_center, focus, k_out,
                      (double2*)E_out, count);
}

sc_status sc_layer_solve(sc_context* ctx, int layers, const double* n, const double* kappa, const double* z,
                         double lambda, int count, const double* k_in, const void* E_in, void* r_E, void* r_k,
                         void* t_E, void* t_k, int* status, void* stream) {
    if (!ctx) {
        set_error("sc_layer_solve: null context");
        return SC_BADINPUT;
    }
    DeviceGuard g(ctx->device);
    return layer_solve(ctx, layers, n, kappa, z, lambda, count, k_in, (const double2*)E_in, (double2*)r_E,
                       (double2*)r_k, (double2*)t_E, (double2*)t_k, status, (cudaStream_t)stream);
}

// ------------------------------------------------------------ host shims
sc_status sc_mkl_eigensolve(void* A, void* evl, void* evt, int N) {
    if (!A || !evl || !evt || N <= 0) {
        set_error("sc_mkl_eigensolve: bad argument");
        return SC_BADINPUT;
    }
    static sc_context* shim_ctx = nullptr;
    static std::mutex mu;
    std::lock_guard<std::mutex> lock(mu);
    if (!shim_ctx) SC_TRY(sc_create(&shim_ctx, 0));
    const size_t bytes = sizeof(double2) * (size_t)N * N;
    double2 *dA, *dV, *dw;
    SC_TRY(shim_ctx->ws.get(&dA, (size_t)N * N, WS_BMAT, 0));
    SC_TRY(shim_ctx->ws.get(&dV, (size_t)N * N, WS_CMAT, 0));
    SC_TRY(shim_ctx->ws.get(&dw, (size_t)N, WS_MU, 0));
    SC_CUDA_TRY(cudaMemcpy(dA, A, bytes, cudaMemcpyHostToDevice));
    sc_status s = sc_eigensolve_batched(shim_ctx, dA, N, 1, dw, dV, nullptr, nullptr);
    if (s != SC_OK && s != SC_NOCONVERGE) return s;
    SC_CUDA_TRY(cudaMemcpy(evt, dV, bytes, cudaMemcpyDeviceToHost));
    SC_CUDA_TRY(cudaMemcpy(evl, dw, sizeof(double2) * N, cudaMemcpyDeviceToHost));
    return s;
}

}  // extern "C"
