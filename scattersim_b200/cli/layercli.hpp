// Shared host flow of scatterlayer and scatterplane: the centre wave, the
// focused beam and the batched layer solve over the C ABI, then the
// coupled-wave structure in the order the reference programs fill it
// (Pi; per boundary l its reflected and transmitted lists).
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <iostream>
#include <string>
#include <vector>

#include "../../include/scattersim_b200.h"
#include "cwio.hpp"

namespace layercli {

using cwio::cplx;

inline int fail(const char* what, sc_status s) {
    std::cerr << "ERROR: " << what << " failed (status " << (int)s << "): " << sc_last_error_string() << std::endl;
    return 1;
}

// FourierWave.h:32-39: E /= sqrt(E.E) (complex squares), then d x (E x d)
inline void orthogonalize(cplx e[3], const double d[3]) {
    const cplx m = std::sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
    for (int i = 0; i < 3; ++i) e[i] /= m;
    const cplx s[3] = {e[1] * d[2] - e[2] * d[1], e[2] * d[0] - e[0] * d[2], e[0] * d[1] - e[1] * d[0]};
    const cplx r[3] = {d[1] * s[2] - d[2] * s[1], d[2] * s[0] - d[0] * s[2], d[0] * s[1] - d[1] * s[0]};
    for (int i = 0; i < 3; ++i) e[i] = r[i];
}

struct Run {
    double lambda = 1.0, alpha = 0.0, beta = 0.0;
    double dir[3] = {0, 0, 1};
    cplx e[3];
    double focus[3] = {0, 0, 0};
    int N0 = 1, N1 = 1;
    std::vector<double> n, kappa, z;   // the padded per-layer lists (L, L-1, L-1)
    int device = 0;
    bool wave_mask[3] = {true, true, true};   // incident, reflected, transmitted lists written
};

// Solve and fill the structure; returns 0 or prints the failure and returns 1.
inline int solve(const Run& r, cwio::CoupledWave& cw) {
    const int L = (int)r.n.size();
    double d[3] = {r.dir[0], r.dir[1], r.dir[2]};
    const double dn = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    if (!(dn > 0)) {
        std::cerr << "ERROR: zero direction" << std::endl;
        return 1;
    }
    for (double& v : d) v /= dn;
    cplx e[3] = {r.e[0], r.e[1], r.e[2]};
    orthogonalize(e, d);
    const double k = 2.0 * M_PI / r.lambda * r.n[0];
    const double kc[3] = {d[0] * k, d[1] * k, d[2] * k};
    sc_context* ctx = nullptr;
    sc_status s;
    if ((s = sc_create(&ctx, r.device)) != SC_OK) return fail("sc_create", s);
    const long long cap = (long long)r.N0 * r.N1;
    const int nb = L - 1;
    double* d_k = nullptr;
    void *d_E = nullptr, *d_out[4] = {};
    if (cudaMalloc(&d_k, sizeof(double) * 3 * cap) != cudaSuccess ||
        cudaMalloc(&d_E, sizeof(cplx) * 3 * cap) != cudaSuccess) {
        std::cerr << "ERROR: device allocation failed" << std::endl;
        return 1;
    }
    for (auto& p : d_out)
        if (nb > 0 && cudaMalloc(&p, sizeof(cplx) * 3 * cap * nb) != cudaSuccess) {
            std::cerr << "ERROR: device allocation failed" << std::endl;
            return 1;
        }
    int count = 0;
    if ((s = sc_beam_polar(ctx, r.alpha, r.beta, r.N0, r.N1, kc, reinterpret_cast<const double*>(e), r.focus, d_k, d_E,
                           &count, nullptr)) != SC_OK)
        return fail("sc_beam_polar", s);
    if ((s = sc_layer_solve(ctx, L, r.n.data(), r.kappa.data(), r.z.data(), r.lambda, count, d_k, d_E, d_out[0],
                            d_out[1], d_out[2], d_out[3], nullptr, nullptr)) != SC_OK)
        return fail("sc_layer_solve", s);
    std::vector<double> hk(3 * (size_t)count);
    std::vector<cplx> hE(3 * (size_t)count), h[4];
    cudaMemcpy(hk.data(), d_k, sizeof(double) * hk.size(), cudaMemcpyDeviceToHost);
    cudaMemcpy(hE.data(), d_E, sizeof(cplx) * hE.size(), cudaMemcpyDeviceToHost);
    for (int q = 0; q < 4; ++q) {
        h[q].resize(3 * (size_t)count * nb);
        if (nb > 0) cudaMemcpy(h[q].data(), d_out[q], sizeof(cplx) * h[q].size(), cudaMemcpyDeviceToHost);
    }
    cw.layers.assign(nb, {});
    for (int t = 0; t < count; ++t) {
        if (r.wave_mask[0]) {
            cwio::Wave w;
            for (int c = 0; c < 3; ++c) {
                w.E[c] = hE[3 * t + c];
                w.k[c] = hk[3 * t + c];
            }
            cw.Pi.push_back(w);
        }
        for (int l = 0; l < nb; ++l) {
            const size_t o = ((size_t)t * nb + l) * 3;
            cwio::Wave wr, wt;
            for (int c = 0; c < 3; ++c) {
                wr.E[c] = h[0][o + c];
                wr.k[c] = h[1][o + c];
                wt.E[c] = h[2][o + c];
                wt.k[c] = h[3][o + c];
            }
            cw.layers[l].z = r.z[l];
            if (r.wave_mask[1]) cw.layers[l].Pr.push_back(wr);
            if (r.wave_mask[2]) cw.layers[l].Pt.push_back(wt);
        }
    }
    cudaFree(d_k);
    cudaFree(d_E);
    for (auto p : d_out) cudaFree(p);
    sc_destroy(ctx);
    return 0;
}

// ScatterLayer.cpp:355-376: one --samples value means a square grid in polar mode
inline void samples(const std::vector<double>& v, int& N0, int& N1) {
    if (v.size() == 1) {
        N0 = N1 = (int)std::sqrt(v[0]);
    } else {
        N0 = (int)v[0];
        N1 = (int)v[1];
    }
}

}  // namespace layercli
