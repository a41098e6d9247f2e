// Internal declarations shared by the scattersim_b200 translation units.
#pragma once

#include <map>
#include <tuple>
#include <vector>

#include "common.cuh"

namespace sc {

// Pooled device workspace owned by a context.  Each slot is a growable buffer
// (stream-ordered cudaMallocAsync/cudaFreeAsync); once warm, no call allocates.
enum WsSlot {
    WS_EIG_TAU = 0, WS_EIG_Z, WS_EIG_Y,
    WS_NF, WS_NIF, WS_OMEGA, WS_BMAT, WS_CMAT, WS_MU, WS_W, WS_CW,
    WS_V, WS_EVL, WS_GD, WS_GC, WS_PIV, WS_INFO, WS_T, WS_T2,
    WS_F, WS_A6, WS_B6, WS_PIV6, WS_TMP, WS_TMP2, WS_BETA, WS_LAT, WS_PZ,
    WS_EVAL_W, WS_EVAL_IDX, WS_STATS,
    WS_HY, WS_HV, WS_HT, WS_HPART, WS_HW, WS_HW2, WS_INV, WS_TREE, WS_GEMV, WS_BINS,
    WS_SWEEP, WS_SWEEP_PTR, WS_OZ_A, WS_OZ_B, WS_OZ_E, WS_OZ_ERR, WS_TUNE_C, WS_TUNE_P,
    WS_LAYER, WS_LAYER_STATUS, WS_MFUN_PTR, WS_MFUN_OUT, WS_CHAIN_T, WS_CRT_RES, WS_FIELD_W, WS_FIELD_T, WS_FIELD_H, WS_FIELD_U, WS_FIELD_HP, WS_FIELD_G, WS_CW_STAGE,
    WS_COUNT
};

struct Workspace {
    void* ptr[WS_COUNT] = {};
    size_t bytes[WS_COUNT] = {};
    // events bracketing the last QR (hqr_kernel) launch, for live roofline timing
    cudaEvent_t ev_hqr[2] = {nullptr, nullptr};
    // per-matrix QR statistics of the last launch: sweeps and phase cycles
    long long* hqr_stats = nullptr;
    int hqr_batch = 0;
    // GEMM autotuner: fastest variant per (m, n, k, batch, slices) shape
    std::map<std::tuple<int, int, int, int, int>, int> gemm_choice;
    // optional per-launch timing of the engine's GEMM kernels (class 0: FP64
    // tensor-pipe tiles, class 1: int8 tcgen05 MMA kernel): event pairs on the
    // launching stream, summed by sc_kernel_stats after the stream has drained
    bool time_kernels = false;
    // modular engine's MMA kernel: 0 = one CTA per 128 x 256 tile, 1 = CTA pairs with 256 x 256 tiles
    int crt_tiles = 0;
    struct KernelMark {
        int cls;
        double flops;      // FP64-equivalent flops of the product (8 m n k per batch entry)
        double int8_ops;   // 2 x int8 multiply-adds issued by the MMA kernel (class 1)
        cudaEvent_t e0, e1;
    };
    std::vector<KernelMark> marks;
    std::vector<cudaEvent_t> event_pool;
    sc_status mark_begin(cudaStream_t st, int cls, double flops, double int8_ops, size_t* id) {
        KernelMark m{cls, flops, int8_ops, nullptr, nullptr};
        for (cudaEvent_t* e : {&m.e0, &m.e1}) {
            if (event_pool.empty()) {
                cudaEvent_t ev;
                cudaError_t r = cudaEventCreate(&ev);
                if (r != cudaSuccess) return cuda_status(r, "cudaEventCreate");
                event_pool.push_back(ev);
            }
            *e = event_pool.back();
            event_pool.pop_back();
        }
        cudaError_t r = cudaEventRecord(m.e0, st);
        if (r != cudaSuccess) return cuda_status(r, "cudaEventRecord");
        marks.push_back(m);
        *id = marks.size() - 1;
        return SC_OK;
    }
    sc_status mark_end(cudaStream_t st, size_t id) {
        cudaError_t r = cudaEventRecord(marks[id].e1, st);
        return r == cudaSuccess ? SC_OK : cuda_status(r, "cudaEventRecord");
    }
    template <typename T>
    sc_status get(T** out, size_t count, int slot, cudaStream_t st) {
        size_t need = count * sizeof(T);
        if (need == 0) need = 16;
        if (bytes[slot] < need) {
            if (ptr[slot]) {
                cudaError_t e = cudaFreeAsync(ptr[slot], st);
                if (e != cudaSuccess) return cuda_status(e, "cudaFreeAsync");
                ptr[slot] = nullptr;
                bytes[slot] = 0;
            }
            size_t alloc = need + need / 8;
            cudaError_t e = cudaMallocAsync(&ptr[slot], alloc, st);
            if (e != cudaSuccess) {
                ptr[slot] = nullptr;
                if (e == cudaErrorMemoryAllocation) {
                    cudaGetLastError();
                    set_error("device allocation of %zu bytes failed", alloc);
                    return SC_OOM;
                }
                return cuda_status(e, "cudaMallocAsync");
            }
            bytes[slot] = alloc;
        }
        *out = reinterpret_cast<T*>(ptr[slot]);
        return SC_OK;
    }
    void release() {
        for (auto& m : marks) {
            cudaEventDestroy(m.e0);
            cudaEventDestroy(m.e1);
        }
        marks.clear();
        for (auto e : event_pool) cudaEventDestroy(e);
        event_pool.clear();
        for (auto& e : ev_hqr)
            if (e) cudaEventDestroy(e);
        ev_hqr[0] = ev_hqr[1] = nullptr;
        for (int i = 0; i < WS_COUNT; ++i) {
            if (ptr[i]) cudaFree(ptr[i]);
            ptr[i] = nullptr;
            bytes[i] = 0;
        }
    }
};

// kernel launch accounting (per process, atomic)
void count_launch(int n = 1);
uint64_t launch_total();

// zgemm.cu
// One batched GEMM C_b = alpha * alpha_b * op(A_b) op(B_b) + beta * C_b.  Each
// operand is addressed either through a device array of per-batch pointers
// (Ap/Bp/Cp, when non-null) or as base + b * stride; alphas (device, per batch)
// is optional.
struct GemmArgs {
    int m = 0, n = 0, k = 0;
    double2 alpha = {1.0, 0.0}, beta = {0.0, 0.0};
    const double2* alphas = nullptr;
    const double2* A = nullptr;
    const double2* const* Ap = nullptr;
    int lda = 1;
    long long sA = 0;
    const double2* B = nullptr;
    const double2* const* Bp = nullptr;
    int ldb = 1;
    long long sB = 0;
    double2* C = nullptr;
    double2* const* Cp = nullptr;
    int ldc = 1;
    long long sC = 0;
};
sc_status zgemm_run(cudaStream_t st, bool conjA, bool conjB, const GemmArgs& g, int batch);
// the FP64 tensor-pipe product with a given CTA tile (64 or 128 rows)
sc_status zgemm_tile(cudaStream_t st, bool conjA, bool conjB, const GemmArgs& g, int batch, int tile);

sc_status zgemm(cudaStream_t st, int m, int n, int k, double2 alpha, const double2* A, int lda,
                long long sA, const double2* B, int ldb, long long sB, double2 beta, double2* C,
                int ldc, long long sC, int batch);

sc_status zgemm_op(cudaStream_t st, bool conjA, bool conjB, int m, int n, int k, double2 alpha,
                   const double2* A, int lda, long long sA, const double2* B, int ldb, long long sB,
                   double2 beta, double2* C, int ldc, long long sC, int batch);

// ozaki.cu: the same product (op = N only) on the int8 tensor cores with
// `slices` 7-bit digits per operand (1..7); err: device word set nonzero if a
// pipeline wait timed out (never cleared here)
sc_status zgemm_ozaki(cudaStream_t st, int slices, const GemmArgs& g, int batch, Workspace& ws, int* err);
// power-of-two row exponents of A (rowexp, batch x m) and column exponents of
// B (colexp, batch x n): max |Re|, |Im| of the row / column < 2^e
sc_status oz_exponents(cudaStream_t st, const GemmArgs& g, int batch, int* rowexp, int* colexp);

// crt.cu: the same product on the int8 tensor cores by modular arithmetic
// (14 moduli, Chinese-remainder reconstruction in FP64); about 2^-47 relative
// to row scale x column scale x k per element for k <= 1250
sc_status zgemm_crt(cudaStream_t st, const GemmArgs& g, int batch, Workspace& ws, int* err);
size_t crt_packed_bytes(int m, int n, int k);
// measured int8 tcgen05 throughput (TOPS) at the modular engine's MMA shape,
// operands resident in shared memory
sc_status int8_peak_probe(int device, Workspace& ws, double* tops);

// A GEMM engine for op = N products: FP64 tensor-pipe tiles, and with
// slices > 0 also int8 digit slices on the tcgen05 tensor cores.  The first
// product of each shape times every candidate once (into scratch output) and
// caches the fastest in the workspace; later products of that shape reuse it.
// force_int8 skips the tuning and runs every product on the digit-slice
// engine; force_crt every product on the modular (CRT) engine.  With
// slices == 7 and neither forced, the modular engine is a tuning candidate too.
struct GemmEngine {
    int slices = 0;
    bool force_int8 = false;
    bool force_crt = false;
    Workspace* ws = nullptr;
    int* err = nullptr;
    sc_status run(cudaStream_t st, const GemmArgs& g, int batch) const;
};

// y = alpha A x + beta y (batched, deterministic two-pass); part: zgemv_part_size entries
sc_status zgemv(cudaStream_t st, int m, int n, double2 alpha, const double2* A, int lda, long long sA,
                const double2* x, long long sx, double2 beta, double2* y, long long sy, int batch, double2* part);
size_t zgemv_part_size(int m, int n, int batch);

// hess.cu: blocked Householder Hessenberg reduction and explicit Q, batched
sc_status hessenberg_blocked(cudaStream_t st, double2* A, int n, int batch, double2* Q, Workspace& ws);

// lu.cu
sc_status getrf(cudaStream_t st, double2* A, int lda, long long sA, int n, int batch, int* ipiv,
                int* info);
sc_status getrs(cudaStream_t st, const double2* LU, int lda, long long sA, int n, const int* ipiv,
                double2* B, int ldb, long long sB, int nrhs, int batch);
sc_status set_identity(cudaStream_t st, double2* B, int ldb, long long sB, int n, int batch);

// eig.cu
size_t hqr_smem_bytes();
sc_status eig_batched(cudaStream_t st, double2* A, int n, int batch, double2* evl, double2* V,
                      int* info, Workspace& ws);
sc_status normalize_columns(cudaStream_t st, double2* V, int rows, int cols, int ld, long long sA,
                            int batch);

// fourier.cu
// R2, Ri2: scratch of Z*S1*Mx entries each; bins: device scratch of Mx + My ints
sc_status fft2_crop(cudaStream_t st, const double2* sample, int Z, int S1, int S2, int Mx, int My,
                    double2* Nf, double2* Nif, double2* R2, double2* Ri2, int* bins);
void crop_bins(int N1, int N2, int M1, int M2, std::vector<int>& rows, std::vector<int>& cols);
sc_status assemble_phi(cudaStream_t st, const double2* Nf, const double2* Nif, int Z, int Mx, int My,
                       const double* lat, double k, double2* Phi);
sc_status assemble_bc(cudaStream_t st, const double2* Nf, const double2* Nif, int Z, int Mx, int My,
                      const double* lat, double k, double2* Bm, double2* Cm);
// L layers of several instances: layer z takes lattice lat + inst[z] * (Mx + My)
// and 1/k^2 = kinv[inst[z]]
sc_status assemble_bc_layers(cudaStream_t st, const double2* Nf, const double2* Nif, int L, int Mx, int My,
                             const double* lat, const int* inst, const double* kinv, double2* Bm, double2* Cm);

// mfun.cu: the inverse layer factor exp(-t_l Phi_l), t_l = i kdz_l, of a batch of
// layers from B, C and Omega = B C (destroyed), in factored form: block l of T
// (stride 4 n2^2) holds F, G B and C G of the half angle (n2 x n2 each, leading
// dimension n2, at offsets 0, n2^2, 2 n2^2).  scr: transfer_scratch_blocks() *
// count * n2^2 entries; dnorm: count doubles; dcoef: count entries.
size_t transfer_scratch_blocks();
sc_status transfer_inv_batched(cudaStream_t st, const GemmEngine& eng, int n2, int count, const double2* B,
                               const double2* C, double2* Om, const std::vector<double>& kdz, double2* T,
                               double2* scr, double* dnorm, double2* dcoef, int* squarings);

// boundary.cu: per-instance blocks of the boundary system (batched over
// instances; order vectors [Sx, Sy, Sz0, Sz1, EF] at svec + b * sv_stride,
// (k, z0) pairs at kz0)
sc_status boundary_f3(cudaStream_t st, int MF, const double2* svec, long long sv_stride, double2* F, long long sF,
                      int count);
sc_status boundary_system(cudaStream_t st, int MF, const double2* svec, long long sv_stride, const double* kz0,
                          double2* A6, long long sA, double2* b6, long long sb, int count);
// the boundary system with R eliminated order by order: 3MF x 3MF in T (needs
// Sz0 != 0 at every order), and x = [R; T] recovered from its solution
sc_status boundary_reduced(cudaStream_t st, int MF, const double2* svec, long long sv_stride, const double* kz0,
                           const double2* const* Y, int ldy, double2* A3, long long sA, double2* b3, long long sb,
                           int count);
sc_status boundary_recover(cudaStream_t st, int MF, const double2* svec, long long sv_stride, const double* kz0,
                           const double2* const* Y, int ldy, const double2* T, long long sT, double2* const* x,
                           int count);
sc_status copy_blocks(cudaStream_t st, int rows, int cols, const double2* const* src, int lds, double2* const* dst,
                      int ldd, int count);

}  // namespace sc
