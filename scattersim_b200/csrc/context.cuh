// Context and host-side plan of a volume solve.
#pragma once

#include <complex>
#include <vector>

#include "kernels.cuh"

struct sc_context {
    int device = 0;
    sc::Workspace ws;
    cudaEvent_t ev[8] = {};
    double stage_ms[8] = {};   // fft assemble eig chain boundary interior | qr | total
    uint64_t launches_at_create = 0;
    int precision = 0;   // SC_SWEEP_* code for the products of sc_volume_solve (sc_volume_precision)
};

namespace sc {

using cplx = std::complex<double>;

constexpr double PI_TRUNC = 3.141592653;   // FourierWave.h:18

// Everything ScatterVolume.cpp computes on the host before the first matrix:
// geometry, polarisation, order choice, lattice (ScatterVolume.cpp:573-685,
// FourierWave.h:319-334).
struct VolumePlan {
    sc_volume_dims dims{};
    int S1 = 0, S2 = 0;
    std::vector<double> z;          // ZL boundary planes
    std::vector<double> up, wq;     // lattice (PI macro), Mx / My
    std::vector<double> UP, WQ;     // Pz lattice (M_PI), Mx / My, without dir*k
    std::vector<cplx> Sx, Sy, Sz0, Sz1;   // column-major order index, MF each
    std::vector<cplx> EF;           // 3 MF
    cplx n_top, n_bot;
};

sc_status make_plan(const sc_volume_params* p, int Z, int S1, int S2, VolumePlan* plan);

}  // namespace sc

namespace sc {

// Focused beam of tira::planewave::SolidAnglePolar and the batched
// homogeneous-layer solve (layer.cu).
sc_status beam_polar(cudaStream_t st, double alpha, double beta, int N0, int N1, const double* kc,
                     const double2* ec, const double* focus, double* kout, double2* Eout, int* count);
sc_status layer_solve(sc_context* ctx, int L, const double* n, const double* kappa, const double* z, double lambda,
                      int count, const double* kin, const double2* Ein, double2* rE, double2* rk, double2* tE,
                      double2* tk, int* status, cudaStream_t st);

}  // namespace sc
