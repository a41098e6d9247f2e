// Layer transfer matrices as matrix functions, batched over layers.
//
// The reference's layer factor GC_i GD_i^-1 (ScatterVolume.cpp:297-335, with
// Ci = exp(i k lambda_j dz) on even and 1/Di = exp(i k lambda_j dz) on odd
// slots) is V exp(t Lambda) V^-1 = exp(t Phi), t = i k dz, for the layer
// matrix Phi = [[0, B], [C, 0]] of volume::phi (FourierWave.h:378-392).  The
// boundary block GD_0 Gc_static^-1 f3 (ScatterVolume.cpp:447) is therefore
//   exp(-t_0 Phi_0) exp(-t_1 Phi_1) ... exp(-t_{L-1} Phi_{L-1}) f3,
// which needs the inverse factors only, and no eigenvectors.  With
// Omega = B C (2M x 2M):
//   exp(-t Phi) = [[ F,        -t G B     ],
//                  [ -t C G,   I + C H B  ]]
//   F = cosh(t sqrt Omega), G = sinh(t sqrt Omega) / (t sqrt Omega),
//   H = (cosh(t sqrt Omega) - I) Omega^-1
// (all three are power series in t^2 Omega, so no square root or inverse is
// formed).  They are evaluated by scaling and double-angle squaring, with the
// scaling s_l chosen per layer:
//   y = (t / 2^s_l)^2 Omega with ||y||_1 <= 4;
//   F = sum_{j<=12} y^j / (2j)!,  G = sum_{j<=12} y^j / (2j+1)!
//   (Paterson-Stockmeyer in y^4: 3 powers + 2 products per series; the
//   truncation error is below 4^13/26! ~ 2e-19 in the 1-norm);
//   s_l - 1 steps of F <- 2 F^2 - I, G <- G F (cosh 2a = 2 cosh^2 a - 1,
//   sinh 2a / 2a = (sinh a / a) cosh a), step j batched over the layers with
//   s_l > j (pointer tables follow each layer's current F and G buffers);
//   the factor is returned at the half angle, in factored form: with F, G of
//   t / 2 (G_t = G F, H_t = (t^2 / 2) G^2 since cosh 2a - 1 = 2 sinh^2 a, and F,
//   G commute as functions of Omega)
//     exp(-t Phi) = [[ 2 F^2 - I,    -t F (G B)             ],
//                    [ -t (C G) F,   I + (t^2/2) (C G)(G B) ]],
//   so a layer is stored as F, G B and C G (three 2M x 2M blocks) and applied
//   to a 4M x 3M vector block X = [X1; X2] by four products:
//     U = (G B) X2, V = F X1, X1' = F (2 V - t U) - X1,
//     X2' = X2 + (C G) ((t^2/2) U - t V)
//   (sweep.cu), which is 32 M^3 fewer multiply-adds per layer than forming the
//   4M x 4M factor and multiplying by it.
// Every product is a batched complex GEMM over all layers of the batch with
// per-layer scalars, run by the caller's GEMM engine (FP64 tensor-pipe tiles,
// or int8 digit slices on the tcgen05 tensor cores).
#include <algorithm>
#include <cmath>
#include <utility>
#include <vector>

#include "common.cuh"
#include "kernels.cuh"

namespace sc {

namespace {

// out_l = c0 I + c1 y + c2 Y2 + c3 Y3 + c4 Y4  (inputs n x n, contiguous, stride n^2;
// out with leading dimension ldo and layer stride so)
__global__ void poly_block_kernel(int n, const double2* __restrict__ y, const double2* __restrict__ Y2,
                                  const double2* __restrict__ Y3, const double2* __restrict__ Y4, double c0,
                                  double c1, double c2, double c3, double c4, double2* __restrict__ out, int ldo,
                                  long long so) {
    const long long nn = (long long)n * n;
    const long long off = (long long)blockIdx.y * nn;
    double2* o = out + (long long)blockIdx.y * so;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nn;
         t += (long long)gridDim.x * blockDim.x) {
        const long long i = off + t;
        double2 v = cscale(y[i], c1);
        v = cadd(v, cscale(Y2[i], c2));
        v = cadd(v, cscale(Y3[i], c3));
        if (c4 != 0.0) v = cadd(v, cscale(Y4[i], c4));
        if (t % (n + 1) == 0) v.x += c0;
        o[(t / n) * ldo + t % n] = v;
    }
}

// P[b] <- 2 P[b] - I for the n x n blocks of a pointer table (leading dimension ld)
__global__ void double_minus_identity_kernel(int n, int ld, double2* const* __restrict__ P) {
    double2* p = P[blockIdx.y];
    const long long nn = (long long)n * n;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nn;
         t += (long long)gridDim.x * blockDim.x) {
        const long long r = t % n, c = t / n;
        double2& v = p[c * ld + r];
        v = make_double2(2.0 * v.x - (r == c ? 1.0 : 0.0), 2.0 * v.y);
    }
}

// A_l *= s_l (real per-layer scale, stored in .x)
__global__ void scale_layers_kernel(long long nn, const double2* __restrict__ s, double2* __restrict__ A) {
    const double f = s[blockIdx.y].x;
    double2* p = A + (long long)blockIdx.y * nn;
    for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < nn;
         t += (long long)gridDim.x * blockDim.x)
        p[t] = cscale(p[t], f);
}

// norm_l = max_c sum_r |A_l(r, c)|  (one CTA per layer, one warp per column)
__global__ void __launch_bounds__(256) norm1_kernel(int n, const double2* __restrict__ A, double* __restrict__ norm) {
    __shared__ double red[8];
    const double2* a = A + (long long)blockIdx.x * n * n;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    double best = 0.0;
    for (int c = w; c < n; c += 8) {
        double s = 0.0;
        for (int r = lane; r < n; r += 32) s += cabs(a[(long long)c * n + r]);
        s = warp_sum(s);
        best = fmax(best, s);
    }
    if (lane == 0) red[w] = best;
    __syncthreads();
    if (threadIdx.x == 0) {
        double m = red[0];
        for (int i = 1; i < 8; ++i) m = fmax(m, red[i]);
        norm[blockIdx.x] = m;
    }
}

unsigned nblocks(long long tot) {
    long long b = (tot + 255) / 256;
    if (b < 1) b = 1;
    if (b > 2048) b = 2048;
    return (unsigned)b;
}

double factorial(int k) {
    double f = 1.0;
    for (int i = 2; i <= k; ++i) f *= i;
    return f;
}

}  // namespace

size_t transfer_scratch_blocks() { return 7; }

sc_status transfer_inv_batched(cudaStream_t st, const GemmEngine& eng, int n2, int count, const double2* B,
                               const double2* C, double2* Om, const std::vector<double>& kdz, double2* T,
                               double2* scr, double* dnorm, double2* dcoef, int* squarings) {
    if (count <= 0) return SC_OK;
    if ((int)kdz.size() != count || n2 <= 0) {
        set_error("transfer_inv_batched: %d layer thicknesses for %d layers", (int)kdz.size(), count);
        return SC_BADINPUT;
    }
    const long long nn = (long long)n2 * n2;
    const long long sT = 4 * nn;   // per-layer block of T (F, G B, C G in its first three quarters)
    double2* Y2 = scr;
    double2* Y3 = scr + (long long)count * nn;
    double2* Y4 = scr + 2LL * count * nn;
    // each layer's G and F stacked as one 2 n2 x n2 block [G; F] (leading dimension 2 n2), so that a
    // double-angle step is one product [G; F] F (F packed once as the right operand); two sets, the
    // second also holding the Paterson-Stockmeyer temporaries P1, P2 of step 3
    const int ls = 2 * n2;
    const long long sS = 2 * nn;
    double2* S0 = scr + 3LL * count * nn;
    double2* S1 = scr + 5LL * count * nn;
    double2* P1 = S1;
    double2* P2 = S1 + (long long)count * nn;

    // 1. scaling per layer: the least s_l >= 1 with (kdz / 2^s_l)^2 ||Omega_l||_1 <= 4
    norm1_kernel<<<count, 256, 0, st>>>(n2, Om, dnorm);
    count_launch();
    SC_CHECK_LAUNCH("norm1");
    std::vector<double> hn(count);
    SC_CUDA_TRY(cudaMemcpyAsync(hn.data(), dnorm, sizeof(double) * count, cudaMemcpyDeviceToHost, st));
    SC_CUDA_TRY(cudaStreamSynchronize(st));
    std::vector<int> sl(count, 1);
    int smax = 1;
    for (int l = 0; l < count; ++l) {
        const double v = kdz[l] * kdz[l] * hn[l];
        if (!std::isfinite(v)) {
            set_error("transfer_inv_batched: non-finite layer matrix norm (layer %d)", l);
            return SC_BADINPUT;
        }
        while (sl[l] < 60 && v / std::ldexp(1.0, 2 * sl[l]) > 4.0) ++sl[l];
        smax = std::max(smax, sl[l]);
    }
    if (squarings) *squarings = smax;

    // per-layer y scale -(kdz / 2^s_l)^2
    std::vector<double2> hc(count);
    for (int l = 0; l < count; ++l) {
        const double h = std::ldexp(kdz[l], -sl[l]);
        hc[l] = make_double2(-h * h, 0.0);
    }
    SC_CUDA_TRY(cudaMemcpyAsync(dcoef, hc.data(), sizeof(double2) * hc.size(), cudaMemcpyHostToDevice, st));
    SC_CUDA_TRY(cudaStreamSynchronize(st));
    const double2* a_y = dcoef;

    const double2 one = make_double2(1.0, 0.0), zero = make_double2(0.0, 0.0);
    auto mm = [&](const double2* A, int lda, long long sA, const double2* Bm, int ldb, long long sB, double2* Cm,
                  int ldc, long long sC, double2 alpha, double2 beta, const double2* alphas) {
        GemmArgs g;
        g.m = n2;
        g.n = n2;
        g.k = n2;
        g.alpha = alpha;
        g.beta = beta;
        g.alphas = alphas;
        g.A = A;
        g.lda = lda;
        g.sA = sA;
        g.B = Bm;
        g.ldb = ldb;
        g.sB = sB;
        g.C = Cm;
        g.ldc = ldc;
        g.sC = sC;
        return eng.run(st, g, count);
    };
    const dim3 ge(nblocks(nn), count);

    // 2. y = (kdz / 2^s_l)^2 * (-1) * Omega, in place
    scale_layers_kernel<<<ge, 256, 0, st>>>(nn, a_y, Om);
    count_launch();
    const double2* y = Om;
    SC_TRY(mm(y, n2, nn, y, n2, nn, Y2, n2, nn, one, zero, nullptr));
    SC_TRY(mm(Y2, n2, nn, y, n2, nn, Y3, n2, nn, one, zero, nullptr));
    SC_TRY(mm(Y2, n2, nn, Y2, n2, nn, Y4, n2, nn, one, zero, nullptr));

    // 3. F and G by Paterson-Stockmeyer in y^4
    for (int which = 0; which < 2; ++which) {
        double c[13];
        for (int j = 0; j <= 12; ++j) c[j] = 1.0 / factorial(2 * j + which);
        double2* out = which ? S0 : S0 + n2;   // G rows, then F rows of the stacked blocks
        poly_block_kernel<<<ge, 256, 0, st>>>(n2, y, Y2, Y3, Y4, c[8], c[9], c[10], c[11], c[12], P1, n2, nn);
        poly_block_kernel<<<ge, 256, 0, st>>>(n2, y, Y2, Y3, Y4, c[4], c[5], c[6], c[7], 0.0, P2, n2, nn);
        poly_block_kernel<<<ge, 256, 0, st>>>(n2, y, Y2, Y3, Y4, c[0], c[1], c[2], c[3], 0.0, out, ls, sS);
        count_launch(3);
        SC_CHECK_LAUNCH("poly_block");
        SC_TRY(mm(Y4, n2, nn, P1, n2, nn, P2, n2, nn, one, one, nullptr));
        SC_TRY(mm(Y4, n2, nn, P2, n2, nn, out, ls, sS, one, one, nullptr));
    }

    // 4. s_l - 1 double-angle steps per layer: [G; F] <- [G F; 2 F^2 - I].  Each
    // layer's current stacked block lives in S0 or S1; step j runs over the
    // layers with s_l > j.
    std::vector<double2*> Sc(count), So(count);
    for (int l = 0; l < count; ++l) {
        Sc[l] = S0 + (long long)l * sS;
        So[l] = S1 + (long long)l * sS;
    }
    std::vector<void*> tab;
    std::vector<std::pair<size_t, int>> steps;   // (table offset, active layers)
    for (int j = 1; j < smax; ++j) {
        std::vector<int> act;
        for (int l = 0; l < count; ++l)
            if (sl[l] > j) act.push_back(l);
        steps.emplace_back(tab.size(), (int)act.size());
        for (int l : act) tab.push_back(Sc[l]);            // [G; F]
        for (int l : act) tab.push_back(Sc[l] + n2);       // F
        for (int l : act) tab.push_back(So[l]);            // [G F; F^2]
        for (int l : act) tab.push_back(So[l] + n2);       // F^2 -> 2 F^2 - I
        for (int l : act) std::swap(Sc[l], So[l]);
    }
    const size_t last = tab.size();
    for (int l = 0; l < count; ++l) tab.push_back(Sc[l]);        // G
    for (int l = 0; l < count; ++l) tab.push_back(Sc[l] + n2);   // F
    void** dtab = nullptr;
    SC_TRY(eng.ws->get(&dtab, tab.size(), WS_MFUN_PTR, st));
    SC_CUDA_TRY(cudaMemcpyAsync(dtab, tab.data(), sizeof(void*) * tab.size(), cudaMemcpyHostToDevice, st));
    auto cp = [&](size_t o) { return reinterpret_cast<const double2* const*>(dtab + o); };
    auto mp = [&](size_t o) { return reinterpret_cast<double2* const*>(dtab + o); };
    // one batched product with any operand given by a pointer table (Ap/Bp/Cp) or by base + stride;
    // m rows, leading dimensions lda / ldb of A and B
    auto mmp = [&](int m, const double2* const* Ap, const double2* A, int lda, long long sA,
                   const double2* const* Bp, const double2* Bm, int ldb, long long sB, double2* const* Cp,
                   double2* Cm, int ldc, long long sC, double2 alpha, double2 beta, const double2* alphas, int batch) {
        GemmArgs g;
        g.m = m;
        g.n = n2;
        g.k = n2;
        g.alpha = alpha;
        g.beta = beta;
        g.alphas = alphas;
        g.Ap = Ap;
        g.A = A;
        g.lda = lda;
        g.sA = sA;
        g.Bp = Bp;
        g.B = Bm;
        g.ldb = ldb;
        g.sB = sB;
        g.Cp = Cp;
        g.C = Cm;
        g.ldc = ldc;
        g.sC = sC;
        return eng.run(st, g, batch);
    };
    for (const auto& sp : steps) {
        const int na = sp.second;
        const size_t sc = sp.first, fc = sc + na, so = fc + na, fo = so + na;
        SC_TRY(mmp(ls, cp(sc), nullptr, ls, 0, cp(fc), nullptr, ls, 0, mp(so), nullptr, ls, 0, one, zero, nullptr,
                   na));                                                                          // [G; F] F
        double_minus_identity_kernel<<<dim3(nblocks(nn), na), 256, 0, st>>>(n2, ls, mp(fo));        // 2 F^2 - I
        count_launch();
        SC_CHECK_LAUNCH("double_minus_identity");
    }

    // 5. the factored layer: F, G B and C G (half angle) into the layer's block of T
    const size_t lg = last, lf = last + count;
    std::vector<void*> outp(count);
    for (int l = 0; l < count; ++l) outp[l] = T + (long long)l * sT;
    void** dout = nullptr;
    SC_TRY(eng.ws->get(&dout, outp.size(), WS_MFUN_OUT, st));
    SC_CUDA_TRY(cudaMemcpyAsync(dout, outp.data(), sizeof(void*) * outp.size(), cudaMemcpyHostToDevice, st));
    SC_TRY(copy_blocks(st, n2, n2, cp(lf), ls, reinterpret_cast<double2* const*>(dout), n2, count));        // F
    SC_TRY(mmp(n2, cp(lg), nullptr, ls, 0, nullptr, B, n2, nn, nullptr, T + nn, n2, sT, one, zero, nullptr,
               count));                                                                                     // G B
    SC_TRY(mmp(n2, nullptr, C, n2, nn, cp(lg), nullptr, ls, 0, nullptr, T + 2 * nn, n2, sT, one, zero, nullptr,
               count));                                                                                     // C G
    return SC_OK;
}

}  // namespace sc
