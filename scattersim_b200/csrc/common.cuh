// Shared device helpers for the scattersim_b200 kernels (sm_100a).
//
// Complex128 values are double2 {re, im}; complex64 values are float2.
// Matrices are column-major with an explicit leading dimension, the layout of
// Eigen::MatrixXcd and of the LAPACK/MKL calls the reference makes
// (third_Lapack.h:37-85).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstdio>

#include "../../include/scattersim_b200.h"

namespace sc {

__host__ __device__ __forceinline__ double2 cmk(double r, double i) { return make_double2(r, i); }
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ double2 cneg(double2 a) { return make_double2(-a.x, -a.y); }
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// a * conj(b)
__host__ __device__ __forceinline__ double2 cmulc(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, a.y * b.y), fma(a.y, b.x, -a.x * b.y));
}
// acc + a * b
__host__ __device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 acc) {
    acc.x = fma(a.x, b.x, acc.x);
    acc.x = fma(-a.y, b.y, acc.x);
    acc.y = fma(a.x, b.y, acc.y);
    acc.y = fma(a.y, b.x, acc.y);
    return acc;
}
__host__ __device__ __forceinline__ double cabs1(double2 a) { return fabs(a.x) + fabs(a.y); }
__host__ __device__ __forceinline__ double cabs(double2 a) { return hypot(a.x, a.y); }
__host__ __device__ __forceinline__ double cnorm2(double2 a) { return a.x * a.x + a.y * a.y; }
// Smith's algorithm for a / b.
__host__ __device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
    if (fabs(b.x) >= fabs(b.y)) {
        double r = b.y / b.x, den = b.x + b.y * r;
        return make_double2((a.x + a.y * r) / den, (a.y - a.x * r) / den);
    } else {
        double r = b.x / b.y, den = b.x * r + b.y;
        return make_double2((a.x * r + a.y) / den, (a.y * r - a.x) / den);
    }
}
// principal square root
__host__ __device__ __forceinline__ double2 csqrt(double2 a) {
    double m = cabs(a);
    if (m == 0.0) return make_double2(0.0, 0.0);
    double t = sqrt(0.5 * (m + fabs(a.x)));
    if (a.x >= 0.0) return make_double2(t, a.y / (2.0 * t));
    return make_double2(fabs(a.y) / (2.0 * t), copysign(t, a.y));
}
// exp(a) for complex a
__host__ __device__ __forceinline__ double2 cexp(double2 a) {
    double e = exp(a.x), s, c;
    sincos(a.y, &s, &c);
    return make_double2(e * c, e * s);
}

__host__ __device__ __forceinline__ float2 fcmul(float2 a, float2 b) {
    return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__host__ __device__ __forceinline__ float2 fcfma(float2 a, float2 b, float2 acc) {
    acc.x = fmaf(a.x, b.x, acc.x);
    acc.x = fmaf(-a.y, b.y, acc.x);
    acc.y = fmaf(a.x, b.y, acc.y);
    acc.y = fmaf(a.y, b.x, acc.y);
    return acc;
}

// Warp and block reductions -------------------------------------------------
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double2 warp_sum2(double2 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
        v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
}

// Sum over the block; `red` must hold >= 32 doubles.  Result valid in all threads.
__device__ __forceinline__ double block_sum(double v, double* red) {
    int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    v = warp_sum(v);
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double r = (lane < nw) ? red[lane] : 0.0;
    r = warp_sum(r);
    return r;
}

// Host-side error plumbing ---------------------------------------------------
void set_error(const char* fmt, ...);
sc_status cuda_status(cudaError_t e, const char* where);

// Dynamic shared memory above 48 KB is granted per kernel and per device (a
// function attribute belongs to the current device's context): raise the
// kernel's limit to `bytes` on the current device unless an earlier call
// there already granted at least that much.  Thread-safe.
sc_status smem_opt_in(const void* kernel, int bytes);
template <typename K>
sc_status smem_opt_in(K* kernel, int bytes) {
    return smem_opt_in(reinterpret_cast<const void*>(kernel), bytes);
}

#define SC_CUDA_TRY(expr)                                                  \
    do {                                                                   \
        cudaError_t _e = (expr);                                           \
        if (_e != cudaSuccess) return ::sc::cuda_status(_e, #expr);        \
    } while (0)

#define SC_TRY(expr)                                                       \
    do {                                                                   \
        sc_status _s = (expr);                                             \
        if (_s != SC_OK) return _s;                                        \
    } while (0)

#define SC_CHECK_LAUNCH(where) SC_CUDA_TRY(cudaGetLastError())

}  // namespace sc
