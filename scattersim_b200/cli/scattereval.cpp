// scattereval: the `scatterview --nogui` slice evaluation of the reference
// (ScatterView.cpp:678-795) over the C ABI's host-buffer shims.
//
//   scattereval --input c.cw [--cuda 0] [--size 100] [--resolution 8]
//               [--axis 1] [--center x y z] [--slice s] [--output xz.npy]
//
// Loads the coupled-wave structure (records read in the reference's record
// frame, E0 rebuilt as tira's getE0() does), unpacks it in cw_unpack order
// (cpuEvaluator.cpp:34-102), evaluates the x-y,
// x-z and y-z slices of N = 2^resolution points with step extent / (N - 1)
// starting at center - extent / 2 (ScatterView.cpp:354-370), and saves the
// slice of --axis (0: y-z at x, 1: x-z at y, 2: x-y at z; the slice
// coordinate is --slice) as an (N, N, 3) complex64 .npy.
#include <chrono>
#include <cmath>
#include <complex>
#include <iostream>

#include "../../include/scattersim_b200.h"
#include "cwio.hpp"

int main(int argc, char** argv) {
    const std::vector<std::string> known = {"input", "help", "cuda", "nogui", "verbose", "size", "resolution",
                                            "output", "axis", "center", "slice", "cw-frame"};
    cwio::Options o;
    try {
        o = cwio::parse(argc, argv, known, "input");
    } catch (const std::exception& e) {
        std::cerr << "ERROR: " << e.what() << std::endl;
        return 1;
    }
    if (o.has("help")) {
        std::cout << "Allowed options:\n  --input arg (=c.cw)\n  --cuda arg (=0)\n  --size arg (=100)\n"
                     "  --resolution arg (=8)\n  --output arg (=xz.npy)\n  --axis arg (=1)\n"
                     "  --center arg (={0, 0, 0})\n  --slice arg (=0)\n"
                     "  --cw-frame arg (=tira) record frame of the file ('tira', 'tira-mirror', 'cartesian', or 'auto': the one that makes the field continuous at the first interface)\n";
        return 1;
    }
    const std::string in = o.str("input", "c.cw"), out = o.str("output", "xz.npy");
    const int device = (int)o.num("cuda", 0), res = (int)o.num("resolution", 8), axis = (int)o.num("axis", 1);
    const float extent = (float)o.num("size", 100.0);
    auto center = o.nums("center", {0, 0, 0});
    const float slice = (float)o.num("slice", 0.0);
    if (center.size() < 3 || axis < 0 || axis > 2 || res < 1 || res > 14) {
        std::cerr << "ERROR: bad --center/--axis/--resolution" << std::endl;
        return 1;
    }
    auto t0 = std::chrono::steady_clock::now();
    cwio::CoupledWave cw;
    try {
        cw = cwio::load_cw(in, cwio::parse_read_frame(o.str("cw-frame", "tira")));
    } catch (const std::exception& e) {
        std::cout << "ERROR: " << e.what() << std::endl;
        return 1;
    }
    // cw_allocate / cw_unpack: Pi, then per layer Pr then Pt; region index
    const int layers = (int)cw.layers.size();
    std::vector<float> zl(layers);
    std::vector<int> begin{0}, end;
    std::vector<std::complex<float>> W;
    auto push = [&](const std::vector<cwio::Wave>& ws) {
        for (auto& w : ws) {
            for (int c = 0; c < 3; ++c) W.push_back(std::complex<float>(w.E[c]));
            for (int c = 0; c < 3; ++c) W.push_back(std::complex<float>(w.k[c]));
        }
    };
    long long total = (long long)cw.Pi.size();
    push(cw.Pi);
    for (int l = 0; l < layers; ++l) {
        zl[l] = (float)cw.layers[l].z;
        total += (long long)cw.layers[l].Pr.size();
        end.push_back((int)total);
        begin.push_back((int)total);
        total += (long long)cw.layers[l].Pt.size();
        push(cw.layers[l].Pr);
        push(cw.layers[l].Pt);
    }
    end.push_back((int)total);
    sc_status s = sc_gpu_initialize(layers, zl.data(), begin.data(), end.data(), W.data(), total, device);
    if (s != SC_OK) {
        std::cerr << "ERROR: sc_gpu_initialize: " << sc_last_error_string() << std::endl;
        return 1;
    }
    const int N = 1 << res;
    const float d = extent / (float)(N - 1);
    const float x0 = (float)center[0] - extent / 2, y0 = (float)center[1] - extent / 2, z0 = (float)center[2] - extent / 2;
    float plane[3] = {0, 0, 0};
    plane[axis] = slice;
    std::vector<std::complex<float>> Exy((size_t)N * N * 3), Exz((size_t)N * N * 3), Eyz((size_t)N * N * 3);
    s = sc_gpu_cw_evaluate(Exy.data(), Exz.data(), Eyz.data(), x0, y0, z0, plane[0], plane[1], plane[2], d, N, device);
    if (s != SC_OK) {
        std::cerr << "ERROR: sc_gpu_cw_evaluate: " << sc_last_error_string() << std::endl;
        return 1;
    }
    double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::cout << "Evaluation (no gui) takes:" << secs << "s" << std::endl;
    const auto& E = axis == 1 ? Exz : (axis == 2 ? Exy : Eyz);
    try {
        cwio::write_npy(out, "<c8", {(size_t)N, (size_t)N, 3}, E.data(), E.size() * sizeof(std::complex<float>));
    } catch (const std::exception& e) {
        std::cerr << "ERROR: " << e.what() << std::endl;
        return 1;
    }
    return 0;
}
