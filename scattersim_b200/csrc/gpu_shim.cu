// Host-buffer shims with the reference's own signatures: gpu_initialize and
// gpu_cw_evaluate (gpuEvaluator.cu:15-26, 131-165).  Like the reference they
// keep one process-wide wave table (set by sc_gpu_initialize) and evaluate
// three N x N slices in float32 with the reference's layer test
// z >= z_l - 0.001; the phase k.r is reduced modulo 2 pi in float64.
#include <mutex>
#include <vector>

#include "kernels.cuh"

namespace sc {
namespace {
struct ShimState {
    int device = -1;
    int layers = 0;
    long long nW = 0;
    float* z = nullptr;
    int* begin = nullptr;
    int* end = nullptr;
    float2* W = nullptr;   // nW x 6 complex64: E0[3], k[3]
    float2* E = nullptr;   // output slice buffer
    size_t Ebytes = 0;
};
ShimState g_shim;
std::mutex g_shim_mu;

// axis 2: x-y at fixed z; axis 1: x-z at fixed y; axis 0: y-z at fixed x
__global__ void slice_kernel(const float2* __restrict__ W, const float* __restrict__ zl,
                             const int* __restrict__ begin, const int* __restrict__ end, int layers, int axis,
                             float a0, float b0, float fixed, float d, int N, float2* __restrict__ out) {
    const int ia = blockIdx.x * blockDim.x + threadIdx.x;
    const int ib = blockIdx.y * blockDim.y + threadIdx.y;
    if (ia >= N || ib >= N) return;
    float x, y, z;
    const float a = a0 + d * ia, b = b0 + d * ib;
    if (axis == 2) { x = a; y = b; z = fixed; }
    else if (axis == 1) { x = a; z = b; y = fixed; }
    else { y = a; z = b; x = fixed; }
    int l = 0;
    for (int li = 0; li < layers; ++li)
        if (z >= zl[li] - 0.001f) l = li + 1;
    float2 e0 = make_float2(0, 0), e1 = make_float2(0, 0), e2 = make_float2(0, 0);
    const double TWO_PI = 6.283185307179586;
    for (int w = begin[l]; w < end[l]; ++w) {
        const float2* p = W + (long long)w * 6;
        const float2 kx = p[3], ky = p[4], kz = p[5];
        const double phr = (double)kx.x * x + (double)ky.x * y + (double)kz.x * z;
        const float phi = kx.y * x + ky.y * y + kz.y * z;
        const double red = phr - TWO_PI * rint(phr * (1.0 / TWO_PI));
        float s, c;
        sincosf((float)red, &s, &c);
        const float amp = expf(-phi);
        const float2 ph = make_float2(amp * c, amp * s);
        e0 = fcfma(p[0], ph, e0);
        e1 = fcfma(p[1], ph, e1);
        e2 = fcfma(p[2], ph, e2);
    }
    const long long o = ((long long)ib * N + ia) * 3;
    out[o] = e0;
    out[o + 1] = e1;
    out[o + 2] = e2;
}
}  // namespace
}  // namespace sc

using namespace sc;

extern "C" {

sc_status sc_gpu_initialize(int layers, const float* z_layers, const int* waves_begin, const int* waves_end,
                            const void* W, long long nW, int device) {
    if (layers < 0 || nW < 0 || (layers > 0 && !z_layers) || !waves_begin || !waves_end || (nW > 0 && !W)) {
        set_error("sc_gpu_initialize: bad argument");
        return SC_BADINPUT;
    }
    for (int l = 0; l <= layers; ++l) {
        if (waves_begin[l] < 0 || waves_end[l] < waves_begin[l] || waves_end[l] > nW) {
            set_error("sc_gpu_initialize: region %d outside the wave table", l);
            return SC_BADINPUT;
        }
    }
    std::lock_guard<std::mutex> lock(g_shim_mu);
    SC_CUDA_TRY(cudaSetDevice(device));
    ShimState& S = g_shim;
    if (S.z) cudaFree(S.z);
    if (S.begin) cudaFree(S.begin);
    if (S.W) cudaFree(S.W);
    S.z = nullptr;
    S.begin = nullptr;
    S.W = nullptr;
    S.device = device;
    S.layers = layers;
    S.nW = nW;
    SC_CUDA_TRY(cudaMalloc(&S.z, sizeof(float) * (layers + 1)));
    SC_CUDA_TRY(cudaMalloc(&S.begin, sizeof(int) * 2 * (layers + 1)));
    S.end = S.begin + layers + 1;
    SC_CUDA_TRY(cudaMalloc(&S.W, sizeof(float2) * 6 * (nW > 0 ? nW : 1)));
    if (layers > 0) SC_CUDA_TRY(cudaMemcpy(S.z, z_layers, sizeof(float) * layers, cudaMemcpyHostToDevice));
    SC_CUDA_TRY(cudaMemcpy(S.begin, waves_begin, sizeof(int) * (layers + 1), cudaMemcpyHostToDevice));
    SC_CUDA_TRY(cudaMemcpy(S.end, waves_end, sizeof(int) * (layers + 1), cudaMemcpyHostToDevice));
    if (nW > 0) SC_CUDA_TRY(cudaMemcpy(S.W, W, sizeof(float2) * 6 * nW, cudaMemcpyHostToDevice));
    return SC_OK;
}

sc_status sc_gpu_cw_evaluate(void* E_xy, void* E_xz, void* E_yz, float x_start, float y_start, float z_start,
                             float x, float y, float z, float d, int N, int device) {
    std::lock_guard<std::mutex> lock(g_shim_mu);
    ShimState& S = g_shim;
    if (!S.W || S.device != device) {
        set_error("sc_gpu_cw_evaluate: sc_gpu_initialize was not called for device %d", device);
        return SC_BADINPUT;
    }
    if (N <= 0 || !E_xy || !E_xz || !E_yz) {
        set_error("sc_gpu_cw_evaluate: bad argument");
        return SC_BADINPUT;
    }
    SC_CUDA_TRY(cudaSetDevice(device));
    const size_t bytes = sizeof(float2) * 3 * (size_t)N * N;
    if (S.Ebytes < bytes) {
        if (S.E) cudaFree(S.E);
        S.E = nullptr;
        S.Ebytes = 0;
        SC_CUDA_TRY(cudaMalloc(&S.E, bytes));
        S.Ebytes = bytes;
    }
    dim3 t(32, 8), g((N + 31) / 32, (N + 7) / 8);
    void* outs[3] = {E_xy, E_xz, E_yz};
    const float a0[3] = {x_start, x_start, y_start};
    const float b0[3] = {y_start, z_start, z_start};
    const float fx[3] = {z, y, x};
    const int axis[3] = {2, 1, 0};
    for (int s = 0; s < 3; ++s) {
        slice_kernel<<<g, t>>>(S.W, S.z, S.begin, S.end, S.layers, axis[s], a0[s], b0[s], fx[s], d, N, S.E);
        count_launch();
        SC_CUDA_TRY(cudaGetLastError());
        SC_CUDA_TRY(cudaMemcpy(outs[s], S.E, bytes, cudaMemcpyDeviceToHost));
    }
    return SC_OK;
}

}  // extern "C"
