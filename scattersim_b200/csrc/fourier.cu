// Fourier coefficients of the permittivity slices and the layer matrices.
//
// fft2_crop replaces fftw_fft2 + fftShift2d (FourierWave.h:82-195) as called
// from volume::phi (FourierWave.h:341, 343).  Only the centred My x Mx block of
// the shifted spectrum survives the crop, so instead of a full FFT the kernels
// evaluate that block directly as a separable partial DFT in FP64:
//   crop index c  ->  FFT bin given by the reference's own shift tables
//                     (crop_bins; bin c - floor(M/2) mod N whenever both
//                     sides of the slice have the same parity),
//   rows pass  R(i, pc) = sum_j A(i,j) w_N2^(fp j)       (Mx bins)
//   cols pass  N(qc,pc) = sum_i R(i,pc) w_N1^(fq i) / (N1 N2)
// with exact twiddles from sincospi on (f j mod N).  A(i, j) is the Eigen
// column-major view of the C-order .npy slice, A(i,j) = flat[i + j*S1]
// (FourierWave.h:283-301).  Both n^2 and (1/n)^2 come out of one read of the
// slice.  The slice is read once per 16 output frequencies (L2-resident).
//
// assemble_phi writes the dense 4M x 4M matrix of volume::phi
// (FourierWave.h:359-394); assemble_bc writes its two non-zero 2M x 2M blocks
// B = Phi[0:2M, 2M:4M] and C = Phi[2M:4M, 0:2M].  The convolution entries use
// the reference's circulant order wrap (FourierWave.h:366-372):
//   row of Nf = ((qi - qj) mod My + My/2) mod My, col likewise in p.
#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace sc {

namespace {
constexpr int RT = 128;     // threads per CTA, rows pass
constexpr int PCH = 16;     // output frequencies per register chunk

__global__ void __launch_bounds__(RT)
dft_rows_kernel(const double2* __restrict__ sample, int S1, int S2, int Mx, const int* __restrict__ bins_x,
                double2* __restrict__ R2, double2* __restrict__ Ri2) {
    extern __shared__ double2 tw[];   // S2 twiddles
    const int z = blockIdx.x;
    for (int t = threadIdx.x; t < S2; t += RT) {
        double s, c;
        sincospi(-2.0 * (double)t / (double)S2, &s, &c);
        tw[t] = make_double2(c, s);
    }
    __syncthreads();
    const int i = blockIdx.y * RT + threadIdx.x;
    if (i >= S1) return;
    const double2* A = sample + (long long)z * S1 * S2;
    double2* r2 = R2 + ((long long)z * S1 + i) * Mx;
    double2* ri2 = Ri2 + ((long long)z * S1 + i) * Mx;
    for (int p0 = 0; p0 < Mx; p0 += PCH) {
        double2 acc[PCH], acci[PCH];
#pragma unroll
        for (int q = 0; q < PCH; ++q) acc[q] = acci[q] = make_double2(0.0, 0.0);
        for (int j = 0; j < S2; ++j) {
            double2 a = A[i + (long long)j * S1];
            double2 e = cmul(a, a);
            double2 inv = cdiv(make_double2(1.0, 0.0), a);
            double2 ei = cmul(inv, inv);
#pragma unroll
            for (int q = 0; q < PCH; ++q) {
                int pc = p0 + q;
                if (pc < Mx) {
                    const int f = bins_x[pc];
                    long long t = ((long long)f * j) % S2;
                    if (t < 0) t += S2;
                    double2 w = tw[t];
                    acc[q] = cfma(e, w, acc[q]);
                    acci[q] = cfma(ei, w, acci[q]);
                }
            }
        }
#pragma unroll
        for (int q = 0; q < PCH; ++q) {
            int pc = p0 + q;
            if (pc < Mx) {
                r2[pc] = acc[q];
                ri2[pc] = acci[q];
            }
        }
    }
}

__global__ void dft_cols_kernel(const double2* __restrict__ R2, const double2* __restrict__ Ri2, int S1,
                                int S2, int Mx, int My, const int* __restrict__ bins_y, double2* __restrict__ Nf,
                                double2* __restrict__ Nif) {
    extern __shared__ double2 tw[];   // S1 twiddles
    const int z = blockIdx.x;
    for (int t = threadIdx.x; t < S1; t += blockDim.x) {
        double s, c;
        sincospi(-2.0 * (double)t / (double)S1, &s, &c);
        tw[t] = make_double2(c, s);
    }
    __syncthreads();
    for (int o = threadIdx.x; o < Mx * My; o += blockDim.x) {
        const int qc = o % My, pc = o / My;
        const int f = bins_y[qc];
        double2 acc = make_double2(0.0, 0.0), acci = make_double2(0.0, 0.0);
        const double2* r2 = R2 + (long long)z * S1 * Mx + pc;
        const double2* ri2 = Ri2 + (long long)z * S1 * Mx + pc;
        for (int i = 0; i < S1; ++i) {
            long long t = ((long long)f * i) % S1;
            if (t < 0) t += S1;
            double2 w = tw[t];
            acc = cfma(r2[(long long)i * Mx], w, acc);
            acci = cfma(ri2[(long long)i * Mx], w, acci);
        }
        // B = B / N1 / N2 (FourierWave.h:186): two divisions, as the reference
        Nf[(long long)z * Mx * My + o] = make_double2(acc.x / S1 / S2, acc.y / S1 / S2);
        Nif[(long long)z * Mx * My + o] = make_double2(acci.x / S1 / S2, acci.y / S1 / S2);
    }
}

// Convolution coefficient for Phi row ri = qi*Mx+pi and column ci = qj*Mx+pj.
__device__ __forceinline__ long long conv_at(int ri, int ci, int Mx, int My) {
    int qi = ri / Mx, pi_ = ri % Mx, qj = ci / Mx, pj = ci % Mx;
    int indR = (qi - qj + My) % My;
    int indC = (pi_ - pj + Mx) % Mx;
    int row = (indR + My / 2) % My, col = (indC + Mx / 2) % Mx;
    return (long long)row + (long long)col * My;
}

// Value of Phi(r, c) (FourierWave.h:378-392); lat = [up (Mx), wq (My)].
__device__ __forceinline__ double2 phi_at(int r, int c, int MF, int Mx, int My, const double2* Nf,
                                          const double2* Nif, const double* up, const double* wq,
                                          double kinv) {
    const int rb = r / MF, ri = r % MF, cb = c / MF, ci = c % MF;
    const double upr = up[ri % Mx], wqr = wq[ri / Mx];
    const double upj = up[ci % Mx], wqj = wq[ci / Mx];
    const bool dg = (ri == ci);
    double2 v = make_double2(0.0, 0.0);
    if (rb == 0) {
        if (cb == 2) v = cscale(cscale(Nif[conv_at(ri, ci, Mx, My)], wqj), upr * kinv);
        else if (cb == 3) {
            v = cscale(cscale(Nif[conv_at(ri, ci, Mx, My)], upj), -upr * kinv);
            if (dg) v.x += 1.0;
        }
    } else if (rb == 1) {
        if (cb == 2) {
            v = cscale(cscale(Nif[conv_at(ri, ci, Mx, My)], wqj), wqr * kinv);
            if (dg) v.x += -1.0;
        } else if (cb == 3) v = cscale(cscale(Nif[conv_at(ri, ci, Mx, My)], upj), -wqr * kinv);
    } else if (rb == 2) {
        if (cb == 0) {
            if (dg) v.x = -upr * wqr * kinv;
        } else if (cb == 1) {
            v = cneg(Nf[conv_at(ri, ci, Mx, My)]);
            if (dg) v.x += upr * upr * kinv;
        }
    } else {
        if (cb == 0) {
            v = Nf[conv_at(ri, ci, Mx, My)];
            if (dg) v.x += -wqr * wqr * kinv;
        } else if (cb == 1) {
            if (dg) v.x = upr * wqr * kinv;
        }
    }
    return v;
}

__global__ void phi_kernel(const double2* __restrict__ Nf, const double2* __restrict__ Nif, int Mx, int My,
                           const double* __restrict__ lat, double kinv, double2* __restrict__ Phi) {
    const int z = blockIdx.y;
    const int MF = Mx * My, n = 4 * MF;
    const long long tot = (long long)n * n;
    const double2* nf = Nf + (long long)z * MF;
    const double2* nif = Nif + (long long)z * MF;
    double2* P = Phi + (long long)z * tot;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x) {
        int r = (int)(t % n), c = (int)(t / n);
        P[t] = phi_at(r, c, MF, Mx, My, nf, nif, lat, lat + Mx, kinv);
    }
}

// B (2M x 2M) = Phi[0:2M, 2M:4M], C = Phi[2M:4M, 0:2M].  Layer z uses the
// lattice and 1/k^2 of instance inst[z] (lat + inst * (Mx + My), kinv_arr)
// when those arrays are given, else the single lattice and kinv.
__global__ void bc_kernel(const double2* __restrict__ Nf, const double2* __restrict__ Nif, int Mx, int My,
                          const double* __restrict__ lat, double kinv, const int* __restrict__ inst,
                          const double* __restrict__ kinv_arr, double2* __restrict__ Bm, double2* __restrict__ Cm) {
    const int z = blockIdx.y;
    const int MF = Mx * My, n = 2 * MF;
    const long long tot = (long long)n * n;
    const double2* nf = Nf + (long long)z * MF;
    const double2* nif = Nif + (long long)z * MF;
    const int ii = inst ? inst[z] : 0;
    const double* L = lat + (long long)ii * (Mx + My);
    const double kv = kinv_arr ? kinv_arr[ii] : kinv;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < tot;
         t += (long long)gridDim.x * blockDim.x) {
        int r = (int)(t % n), c = (int)(t / n);
        Bm[(long long)z * tot + t] = phi_at(r, c + n, MF, Mx, My, nf, nif, L, L + Mx, kv);
        Cm[(long long)z * tot + t] = phi_at(r + n, c, MF, Mx, My, nf, nif, L, L + Mx, kv);
    }
}
}  // namespace

// FFT bins that land in the cropped block: the index tables of fftShift2d
// (FourierWave.h:82-145) for an N1 x N2 matrix, offset by the crop origin
// (N1/2 - M1/2, N2/2 - M2/2) of FourierWave.h:194.  The shift amounts of both
// axes follow the parity of N1, so an even x odd slice gets the reference's
// irregular column table, reproduced here as is.
void crop_bins(int N1, int N2, int M1, int M2, std::vector<int>& rows, std::vector<int>& cols) {
    int p, q;
    if (N1 % 2 == 1) {
        p = N1 / 2;
        q = N2 / 2;
    } else {
        p = (N1 + 1) / 2;
        q = (N2 + 1) / 2;
    }
    std::vector<int> indx(N1), indy(N2);
    if (N1 % 2 == 1) {
        for (int i = 0; i < N1 - p - 1; ++i) indx[i] = (N1 - p) + i;
        for (int i = (N1 - p - 1 > 0 ? N1 - p - 1 : 0); i < N1; ++i) indx[i] = i - (N1 - p - 1);
    } else {
        for (int i = 0; i < N1 - p; ++i) indx[i] = p + i;
        for (int i = N1 - p; i < N1; ++i) indx[i] = i - (N1 - p);
    }
    if (N2 % 2 == 1) {
        for (int i = 0; i < N2 - q - 1; ++i) indy[i] = (N2 - q) + i;
        for (int i = (N2 - q - 1 > 0 ? N2 - q - 1 : 0); i < N2; ++i) indy[i] = i - (N2 - q - 1);
    } else {
        for (int i = 0; i < N2 - q; ++i) indy[i] = q + i;
        for (int i = N2 - q; i < N2; ++i) indy[i] = i - (N2 - q);
    }
    rows.resize(M1);
    cols.resize(M2);
    for (int i = 0; i < M1; ++i) rows[i] = indx[N1 / 2 - M1 / 2 + i];
    for (int j = 0; j < M2; ++j) cols[j] = indy[N2 / 2 - M2 / 2 + j];
}

sc_status fft2_crop(cudaStream_t st, const double2* sample, int Z, int S1, int S2, int Mx, int My,
                       double2* Nf, double2* Nif, double2* R2, double2* Ri2, int* bins) {
    if (Z <= 0 || S1 <= 0 || S2 <= 0 || Mx <= 0 || My <= 0 || Mx > S2 || My > S1) {
        set_error("fft2_crop: bad sizes Z=%d S1=%d S2=%d Mx=%d My=%d", Z, S1, S2, Mx, My);
        return SC_BADINPUT;
    }
    if ((size_t)(S1 > S2 ? S1 : S2) * sizeof(double2) > 200 * 1024) {
        set_error("fft2_crop: slice side too large for the twiddle table");
        return SC_BADINPUT;
    }
    SC_CUDA_TRY(cudaFuncSetAttribute(dft_rows_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    SC_CUDA_TRY(cudaFuncSetAttribute(dft_cols_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
    std::vector<int> by, bx;
    crop_bins(S1, S2, My, Mx, by, bx);
    std::vector<int> hb(bx);
    hb.insert(hb.end(), by.begin(), by.end());
    SC_CUDA_TRY(cudaMemcpyAsync(bins, hb.data(), sizeof(int) * hb.size(), cudaMemcpyHostToDevice, st));
    dim3 g1(Z, (S1 + RT - 1) / RT);
    dft_rows_kernel<<<g1, RT, S2 * sizeof(double2), st>>>(sample, S1, S2, Mx, bins, R2, Ri2);
    count_launch();
    dft_cols_kernel<<<Z, 256, S1 * sizeof(double2), st>>>(R2, Ri2, S1, S2, Mx, My, bins + Mx, Nf, Nif);
    count_launch();
    SC_CHECK_LAUNCH("fft2_crop");
    return SC_OK;
}

sc_status assemble_phi(cudaStream_t st, const double2* Nf, const double2* Nif, int Z, int Mx, int My,
                       const double* lat, double k, double2* Phi) {
    const long long n = 4LL * Mx * My;
    long long blocks = (n * n + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    dim3 g((unsigned)blocks, Z);
    phi_kernel<<<g, 256, 0, st>>>(Nf, Nif, Mx, My, lat, 1.0 / (k * k), Phi);
    count_launch();
    SC_CHECK_LAUNCH("assemble_phi");
    return SC_OK;
}

sc_status assemble_bc(cudaStream_t st, const double2* Nf, const double2* Nif, int Z, int Mx, int My,
                      const double* lat, double k, double2* Bm, double2* Cm) {
    const long long n = 2LL * Mx * My;
    long long blocks = (n * n + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    dim3 g((unsigned)blocks, Z);
    bc_kernel<<<g, 256, 0, st>>>(Nf, Nif, Mx, My, lat, 1.0 / (k * k), nullptr, nullptr, Bm, Cm);
    count_launch();
    SC_CHECK_LAUNCH("assemble_bc");
    return SC_OK;
}

sc_status assemble_bc_layers(cudaStream_t st, const double2* Nf, const double2* Nif, int L, int Mx, int My,
                             const double* lat, const int* inst, const double* kinv, double2* Bm, double2* Cm) {
    const long long n = 2LL * Mx * My;
    long long blocks = (n * n + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    if (L <= 0) return SC_OK;
    dim3 g((unsigned)blocks, L);
    bc_kernel<<<g, 256, 0, st>>>(Nf, Nif, Mx, My, lat, 0.0, inst, kinv, Bm, Cm);
    count_launch();
    SC_CHECK_LAUNCH("assemble_bc_layers");
    return SC_OK;
}

}  // namespace sc
