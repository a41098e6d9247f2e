// scattervolume / scatterthinvolume: the reference's command line over the C ABI.
//
// Same long options and defaults as ScatterVolume.cpp:511-529 (--sample,
// --lambda, --direction, --ex, --ey, --ez, --n, --kappa, --size, --z,
// --output, --coef, --psf, --external, --log, --npz), reads the complex128
// .npy sample, solves on the GPU through libscattersim_b200 and writes the
// coupled-wave structure (.cw).  The stdout summary follows
// ScatterVolume.cpp:995-1002.  scatterthinvolume is the same program (a 2-D
// sample is one layer, FourierWave.h:291-299).
//
// Records are stored in the reference's record frame (--cw-frame tira, the
// default: the E0 pair in the frame rotated to Re k); --cw-frame tira-mirror
// stores a downward wave's pair in the frame of its z-mirrored direction (the
// frame of the waves tira::planewave's constructor makes, which the reference
// uses for these waves); --cw-frame cartesian stores (E_x, E_y).
#include <cuda_runtime.h>

#include <chrono>
#include <cmath>
#include <ctime>
#include <iostream>

#include "../../include/scattersim_b200.h"
#include "cwio.hpp"

using cwio::cplx;

namespace {

int fail(const char* what, sc_status s) {
    std::cerr << "ERROR: " << what << " failed (status " << (int)s << "): " << sc_last_error_string() << std::endl;
    return 1;
}

}  // namespace

int main(int argc, char** argv) {
    const std::vector<std::string> known = {"help", "sample", "lambda", "direction", "ex", "ey", "ez", "n", "kappa",
                                            "size", "z", "output", "coef", "psf", "external", "log", "npz",
                                            "cw-frame", "cuda"};
    cwio::Options o;
    try {
        o = cwio::parse(argc, argv, known);
    } catch (const std::exception& e) {
        std::cerr << "ERROR: " << e.what() << std::endl;
        return 1;
    }
    if (o.has("help")) {
        std::cout << "Allowed options:\n"
                     "  --help                 produce help message\n"
                     "  --sample arg           input sample as an .npy file\n"
                     "  --lambda arg (=1)      incident field vacuum wavelength\n"
                     "  --direction arg (=0, 0, 1) incoming field direction\n"
                     "  --ex arg (=0, 0)       x component of the electrical field\n"
                     "  --ey arg (=1, 0)       y component of the electrical field\n"
                     "  --ez arg (=0 0)        z component of the electrical field\n"
                     "  --n arg (=1, 1)        real refractive index of the upper and lower layers\n"
                     "  --kappa arg (=0.00)    absorbance of the lower layer\n"
                     "  --size arg (=10, 10, 4) the real size of the sample\n"
                     "  --z arg (=0.0)         the center of the sample along z-axis\n"
                     "  --output arg (=c.cw)   output filename for the coupled wave structure\n"
                     "  --coef arg             number of Fourier coefficients (1 or 2 values)\n"
                     "  --psf                  all Fourier orders of the incident field set to E0\n"
                     "  --external             save waves for the external field only\n"
                     "  --log                  produce a log file\n"
                     "  --npz                  calculate Px and Py only\n"
                     "  --cw-frame arg (=tira)  E pair stored in the record frame ('tira'; 'tira-mirror': downward waves in the\n"
                     "                         frame of their z-mirrored direction) or as (E_x, E_y) ('cartesian')\n"
                     "  --cuda arg (=0)        CUDA device\n";
        return 1;
    }
    sc_volume_params p;
    sc_volume_params_default(&p);
    p.lambda = o.num("lambda", 1.0);
    auto dir = o.nums("direction", {0, 0, 1});
    auto ex = o.nums("ex", {0, 0}), ey = o.nums("ey", {1, 0}), ez = o.nums("ez", {0, 0});
    auto n = o.nums("n", {1, 1}), size = o.nums("size", {10, 10, 2}), coef = o.nums("coef", {});
    auto kap = o.nums("kappa", {0});
    if (dir.size() < 3 || ex.size() < 2 || ey.size() < 2 || ez.size() < 2 || n.size() < 2 || size.size() < 3) {
        std::cerr << "ERROR: --direction/--size take 3 values, --ex/--ey/--ez/--n take 2" << std::endl;
        return 1;
    }
    for (int i = 0; i < 3; ++i) {
        p.direction[i] = dir[i];
        p.size[i] = size[i];
    }
    for (int i = 0; i < 2; ++i) {
        p.ex[i] = ex[i];
        p.ey[i] = ey[i];
        p.ez[i] = ez[i];
        p.n[i] = n[i];
    }
    p.kappa = kap.empty() ? 0.0 : kap[0];
    p.z = o.num("z", 0.0);
    p.ncoef = (int)(coef.size() > 2 ? 2 : coef.size());
    for (int i = 0; i < p.ncoef; ++i) p.coef[i] = (int)coef[i];
    p.psf = o.has("psf");
    p.external = o.has("external");
    p.npz = o.has("npz");
    const std::string out = o.str("output", "c.cw");
    cwio::Frame frame;
    try {
        frame = cwio::parse_frame(o.str("cw-frame", "tira"));
    } catch (const std::exception& e) {
        std::cerr << "ERROR: " << e.what() << std::endl;
        return 1;
    }
    if (!o.has("sample")) {
        std::cerr << "ERROR: no --sample given" << std::endl;
        return 1;
    }
    cwio::NpyArray smp;
    try {
        smp = cwio::read_npy(o.str("sample", ""));
    } catch (const std::exception& e) {
        std::cerr << "ERROR: " << e.what() << std::endl;
        return 1;
    }
    if (smp.descr != "<c16" || (smp.shape.size() != 2 && smp.shape.size() != 3)) {
        std::cerr << "ERROR: the sample must be a 2-D or 3-D complex128 array" << std::endl;
        return 1;
    }
    const int Z = smp.shape.size() == 3 ? (int)smp.shape[0] : 1;
    const int S1 = (int)smp.shape[smp.shape.size() - 2], S2 = (int)smp.shape[smp.shape.size() - 1];
    auto t0 = std::chrono::steady_clock::now();

    sc_volume_dims dims;
    sc_status s = sc_volume_plan(&p, Z, S1, S2, &dims);
    if (s != SC_OK) return fail("sc_volume_plan", s);
    if (dims.clamped) {
        std::cout << "Cutting off invalid waves with imagnery sz..." << std::endl;
        std::cout << "[WARNING] Propagation directions for decomposed waves are not all downward." << std::endl;
    }
    sc_context* ctx = nullptr;
    if ((s = sc_create(&ctx, (int)o.num("cuda", 0))) != SC_OK) return fail("sc_create", s);
    const int MF = dims.MF;
    void *d_smp = nullptr, *d_x = nullptr, *d_evl = nullptr, *d_qc = nullptr, *d_qh = nullptr;
    const size_t qbytes = sizeof(cplx) * (size_t)Z * 3 * MF * 2 * MF;
    if (cudaMalloc(&d_smp, smp.data.size()) != cudaSuccess || cudaMalloc(&d_x, sizeof(cplx) * 6 * MF) != cudaSuccess ||
        cudaMalloc(&d_evl, sizeof(cplx) * Z * 4 * MF) != cudaSuccess ||
        (!p.external && (cudaMalloc(&d_qc, qbytes) != cudaSuccess || cudaMalloc(&d_qh, qbytes) != cudaSuccess))) {
        std::cerr << "ERROR: device allocation failed" << std::endl;
        return 1;
    }
    cudaMemcpy(d_smp, smp.data.data(), smp.data.size(), cudaMemcpyHostToDevice);
    int info = 0;
    s = sc_volume_solve(ctx, &p, d_smp, Z, S1, S2, d_x, d_evl, d_qc, d_qh, &info, nullptr);
    if (s != SC_OK) return fail("sc_volume_solve", s);
    long long nw = 0;
    std::vector<int> begin(Z + 2), end(Z + 2);
    std::vector<double> zl(Z + 1);
    if ((s = sc_volume_waves(ctx, &p, Z, S1, S2, nullptr, nullptr, nullptr, nullptr, 0, &nw, begin.data(), end.data(),
                             zl.data(), nullptr, nullptr, nullptr)) != SC_OK)
        return fail("sc_volume_waves", s);
    void *d_E = nullptr, *d_k = nullptr;
    if (cudaMalloc(&d_E, sizeof(cplx) * 3 * nw) != cudaSuccess || cudaMalloc(&d_k, sizeof(cplx) * 3 * nw) != cudaSuccess) {
        std::cerr << "ERROR: device allocation of the wave table failed" << std::endl;
        return 1;
    }
    if ((s = sc_volume_waves(ctx, &p, Z, S1, S2, d_x, d_evl, d_qc, d_qh, 0, &nw, begin.data(), end.data(), zl.data(),
                             d_E, d_k, nullptr)) != SC_OK)
        return fail("sc_volume_waves", s);
    // the file straight from the device table (table order = file order: Pi,
    // then per boundary its Pr and its Pt list); list sizes of
    // CoupledWaveStructure (ScatterVolume.cpp:907-987): boundary 0 reflects MF
    // waves, the last transmits MF, interior lists hold 2 MF^2 modes
    const long long interior = p.external ? 0 : 2LL * MF * MF;
    std::vector<long long> counts(1 + 2 * (Z + 1));
    counts[0] = MF;
    long long pos = MF;
    for (int l = 0; l <= Z; ++l) {
        counts[1 + 2 * l] = (l == 0) ? MF : interior;
        counts[2 + 2 * l] = (l == Z) ? MF : interior;
        pos += counts[1 + 2 * l] + counts[2 + 2 * l];
    }
    if (pos != nw) {
        std::cerr << "ERROR: wave table size mismatch" << std::endl;
        return 1;
    }
    if (!out.empty()) {
        if ((s = sc_cw_write(ctx, out.c_str(), d_E, d_k, nw, Z + 1, zl.data(), counts.data(),
                             frame == cwio::Frame::tira ? 0 : (frame == cwio::Frame::cartesian ? 1 : 2),
                             nullptr)) != SC_OK)
            return fail("sc_cw_write", s);
    }
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::cout << "Field saved in " << out << "." << std::endl;
    std::cout << "Number of pixels (x, y): [" << S2 << "," << S1 << "]" << std::endl;
    std::cout << "Number of sublayers: " << Z << std::endl;
    std::cout << "Number of Fourier coefficients (Mx, My): [" << dims.Mx << "," << dims.My << "]" << std::endl;
    std::cout << "Effective number of Fourier coefficients: [" << MF << "]" << std::endl;
    if (o.has("log")) {
        std::string name = std::to_string((long long)std::time(nullptr)) + "_scattervolume.log";
        std::FILE* f = std::fopen(name.c_str(), "w");
        if (f) {
            double ms[8];
            sc_volume_stage_ms(ctx, ms);
            for (int c = 0; c < argc; ++c) std::fprintf(f, "%s ", argv[c]);
            std::fprintf(f, "\nstage ms: fft %.3f assemble %.3f eig %.3f chain %.3f boundary %.3f interior %.3f\n",
                         ms[0], ms[1], ms[2], ms[3], ms[4], ms[5]);
            std::fprintf(f, "Total time: %.6f s\n", secs);
            std::fclose(f);
        }
    }
    cudaFree(d_E);
    cudaFree(d_k);
    cudaFree(d_smp);
    cudaFree(d_x);
    cudaFree(d_evl);
    cudaFree(d_qc);
    cudaFree(d_qh);
    sc_destroy(ctx);
    return 0;
}
