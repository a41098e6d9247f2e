// Allocation-free batched linear solve.
//
// sc_linearsolve_batched_noalloc solves A X = B exactly like
// sc_linearsolve_batched (same LU kernels, same results) but allocates no
// device memory.  It is for callers that cannot call cudaMalloc: real-time
// loops that must not take the implicit device-wide synchronisation of
// cudaMalloc/cudaFree, and host programs (a solver plugin inside a larger
// application, say) whose framework reserves the GPU's memory up front and
// forbids further device allocations, so that a late cudaMalloc would stall
// other work or fail with out-of-memory in the middle of a run.  Those callers
// pass in A, B and info and get the same solve without a context.
//
// Its only scratch -- the pivot indices and one status word per system --
// lives in g_noalloc_scratch, a fixed array in this library's device memory
// (NOALLOC_MAX_PIVOTS + NOALLOC_MAX_BATCH ints, 260 KiB).  Every GPU that loads
// the library's device code holds that array until the process exits.
//
// In host code the array's name is only a host-side stand-in for the symbol,
// not a device address: passed to a kernel it would fault or, where the GPU
// can reach host memory, silently address the wrong memory.  The device
// address is therefore looked up with cudaGetSymbolAddress once per device,
// with that device current, on the first call made on that device; that first
// call should come before any stream capture starts.  The looked-up address is
// kept for the life of the process: after cudaDeviceReset the library's
// module is reloaded and the kept address is stale, so do not call this entry
// point after resetting the device.
//
// Each call ends by copying the status words back to the host and
// synchronising `stream` (info is a host array, as in the allocating entry),
// except while `stream` is capturing into a CUDA graph: a capture accepts
// neither a copy into pageable host memory nor a synchronisation, so the call
// then records only its clear of the status words and its LU kernels (no
// allocation, and no other driver call once a first call on the device has
// looked up the array and raised the kernels' shared-memory limits), leaves
// info untouched and returns SC_OK; each replay of the graph solves again.
//
// All calls share the one array and keep the last call's contents: the status
// words are cleared on the stream at the start of every call, and calls whose
// work overlaps on the GPU (different streams, or different host threads
// without ordering) race on the array.
#include <mutex>

#include "kernels.cuh"

namespace {
constexpr int NOALLOC_MAX_PIVOTS = 65536;   // n * batch
constexpr int NOALLOC_MAX_BATCH = 1024;
constexpr int MAX_DEVICES = 64;

static __device__ __align__(256) int g_noalloc_scratch[NOALLOC_MAX_PIVOTS + NOALLOC_MAX_BATCH];

int* g_scratch_addr[MAX_DEVICES] = {};
std::mutex g_scratch_mu;
}  // namespace

using namespace sc;

extern "C" sc_status sc_linearsolve_batched_noalloc(void* A, int n, void* B, int nrhs, int batch, int* info,
                                                    void* stream) {
    if (!A || !B || n <= 0 || nrhs <= 0 || batch <= 0) {
        set_error("sc_linearsolve_batched_noalloc: bad argument");
        return SC_BADINPUT;
    }
    if (batch > NOALLOC_MAX_BATCH || (long long)n * batch > NOALLOC_MAX_PIVOTS) {
        set_error("sc_linearsolve_batched_noalloc: n*batch = %lld (batch %d) exceeds the fixed scratch "
                  "(n*batch <= %d, batch <= %d)",
                  (long long)n * batch, batch, NOALLOC_MAX_PIVOTS, NOALLOC_MAX_BATCH);
        return SC_BADINPUT;
    }
    int dev = 0;
    SC_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= MAX_DEVICES) {
        set_error("sc_linearsolve_batched_noalloc: device %d out of range", dev);
        return SC_BADINPUT;
    }
    if (stream) {
        int sdev = dev;
        SC_CUDA_TRY(cudaStreamGetDevice((cudaStream_t)stream, &sdev));
        if (sdev != dev) {
            set_error("sc_linearsolve_batched_noalloc: the stream belongs to device %d, the current device is %d",
                      sdev, dev);
            return SC_BADINPUT;
        }
    }
    int* base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_scratch_mu);
        if (!g_scratch_addr[dev]) {
            void* p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
            if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
            g_scratch_addr[dev] = static_cast<int*>(p);
        }
        base = g_scratch_addr[dev];
    }
    int* piv = base;
    int* dinfo = base + NOALLOC_MAX_PIVOTS;
    cudaStream_t st = (cudaStream_t)stream;
    cudaStreamCaptureStatus capture = cudaStreamCaptureStatusNone;
    SC_CUDA_TRY(cudaStreamIsCapturing(st, &capture));
    // the previous call's status words are still in the array
    SC_CUDA_TRY(cudaMemsetAsync(dinfo, 0, sizeof(int) * batch, st));
    const long long sA = (long long)n * n, sB = (long long)n * nrhs;
    SC_TRY(getrf(st, (double2*)A, n, sA, n, batch, piv, dinfo));
    SC_TRY(getrs(st, (const double2*)A, n, sA, n, piv, (double2*)B, n, sB, nrhs, batch));
    if (capture != cudaStreamCaptureStatusNone) return SC_OK;   // recorded into the caller's graph
    int hinfo[NOALLOC_MAX_BATCH];
    SC_CUDA_TRY(cudaMemcpyAsync(hinfo, dinfo, sizeof(int) * batch, cudaMemcpyDeviceToHost, st));
    SC_CUDA_TRY(cudaStreamSynchronize(st));
    int bad = 0;
    for (int b = 0; b < batch; ++b) {
        if (info) info[b] = hinfo[b];
        if (hinfo[b]) bad = 1;
    }
    if (bad) {
        set_error("sc_linearsolve_batched_noalloc: exactly singular matrix");
        return SC_SINGULAR;
    }
    return SC_OK;
}
