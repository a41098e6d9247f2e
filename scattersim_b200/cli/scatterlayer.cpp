// scatterlayer: the reference's homogeneous-multilayer program over the C ABI.
//
// Same long options and defaults as ScatterLayer.cpp:285-303 (--lambda,
// --direction, --ex, --ey, --ez, --n, --kappa, --z, --output_sample, --output,
// --alpha, --beta, --na, --samples, --mode, --log), the same layer padding
// (:328-343), focused beam (polar mode, :355-385) and one solve per incident
// wave (:390-420) -- here one batched GPU launch for the whole beam -- and the
// same .cw layout (records in the reference's record frame) plus the
// homogeneous sample .npy of the internal layers (:426-434) for scattervolume.
// --mode montecarlo is refused: its random sampler (tira) is not available.
#include <chrono>
#include <cmath>
#include <iostream>

#include "layercli.hpp"

int main(int argc, char** argv) {
    const std::vector<std::string> known = {"help", "lambda", "direction", "ex", "ey", "ez", "n", "kappa", "z",
                                            "output_sample", "output", "alpha", "beta", "na", "samples", "mode",
                                            "log", "cuda", "cw-frame"};
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
                     "  --lambda arg (=1)      incident field vacuum wavelength\n"
                     "  --direction arg (=0, 0, 1) incoming field direction\n"
                     "  --ex arg (=0, 0)       x component of the electrical field\n"
                     "  --ey arg (=1, 0)       y component of the electrical field\n"
                     "  --ez arg (=0 0)        z component of the electrical field\n"
                     "  --n arg (=1, 1.4, 1.4, 1.0) real refractive index (optical path length) of all L layers\n"
                     "  --kappa arg (=0.05, 0.00, 0.00) absorbance of layers 2+ (layer 1 is always 0.0)\n"
                     "  --z arg (=-5.0, 0.0, 5.0) position of each layer boundary\n"
                     "  --output_sample arg (=sample.npy) output the sample as the input for scattervolume\n"
                     "  --output arg (=a.cw)   output filename for the coupled wave structure\n"
                     "  --alpha arg (=1)       angle used to focus the incident field\n"
                     "  --beta arg (=0)        internal obscuration angle (for simulating reflective optics)\n"
                     "  --na arg               focus angle expressed as a numerical aperture (overrides --alpha)\n"
                     "  --samples arg (=64 64) number of samples (can be specified in 2 dimensions)\n"
                     "  --mode arg (=polar)    sampling mode (polar)\n"
                     "  --cw-frame arg (=tira) record frame of the written .cw ('tira', 'tira-mirror' or 'cartesian')\n";
        return 1;
    }
    auto t0 = std::chrono::steady_clock::now();
    layercli::Run r;
    r.lambda = o.num("lambda", 1.0);
    auto dir = o.nums("direction", {0, 0, 1});
    auto ex = o.nums("ex", {0, 0}), ey = o.nums("ey", {1, 0}), ez = o.nums("ez", {0, 0});
    if (dir.size() < 3 || ex.size() < 2 || ey.size() < 2 || ez.size() < 2) {
        std::cerr << "ERROR: --direction takes 3 values, --ex/--ey/--ez 2" << std::endl;
        return 1;
    }
    for (int i = 0; i < 3; ++i) r.dir[i] = dir[i];
    r.e[0] = {ex[0], ex[1]};
    r.e[1] = {ey[0], ey[1]};
    r.e[2] = {ez[0], ez[1]};
    std::vector<double> n = o.nums("n", {1, 1.4, 1.4, 1.0}), kappa = o.nums("kappa", {0.05}),
                        z = o.nums("z", {-5.0, 0.0, 5.0});
    if (n.empty()) {
        std::cerr << "ERROR: --n needs at least one value" << std::endl;
        return 1;
    }
    // layer count and padding (ScatterLayer.cpp:328-343)
    size_t L = n.size();
    if (kappa.size() + 1 > L) L = kappa.size() + 1;
    if (z.size() + 1 > L) L = z.size() + 1;
    n.resize(L, n.back());
    kappa.resize(L - 1, 0.0);
    if (z.empty() && L > 1) z.push_back(0.0);
    while (z.size() + 1 < L) z.push_back(z.back() + 10.0);
    z.resize(L - 1);
    r.n = n;
    r.kappa = kappa;
    r.z = z;
    r.alpha = o.num("alpha", 1.0);
    r.beta = o.num("beta", 0.0);
    if (o.has("na")) r.alpha = std::asin(o.num("na", 0.0) / n[0]);          // :324-326
    layercli::samples(o.nums("samples", {64, 64}), r.N0, r.N1);
    if (o.str("mode", "polar") != "polar") {
        std::cerr << "ERROR: only --mode polar is supported (the Monte Carlo sampler's generator is not available)"
                  << std::endl;
        return 1;
    }
    if (r.alpha == 0.0) r.N0 = r.N1 = 1;                                      // :373-376
    r.device = (int)o.num("cuda", 0);
    cwio::Frame frame;
    try {
        frame = cwio::parse_frame(o.str("cw-frame", "tira"));
    } catch (const std::exception& e) {
        std::cerr << "ERROR: " << e.what() << std::endl;
        return 1;
    }
    cwio::CoupledWave cw;
    if (layercli::solve(r, cw)) return 1;
    const std::string out = o.str("output", "a.cw"), smp = o.str("output_sample", "sample.npy");
    try {
        if (!out.empty()) cwio::save_cw(out, cw, frame);
        if (!smp.empty() && L >= 3) {
            // the internal layers as a (L-2, 1, 1) complex128 volume (:426-434)
            std::vector<cwio::cplx> ref(L - 2);
            for (size_t i = 0; i + 2 < L; ++i) ref[i] = cwio::cplx(n[i + 1], kappa[i]);
            cwio::write_npy(smp, "<c16", {L - 2, 1, 1}, ref.data(), sizeof(cwio::cplx) * ref.size());
        }
    } catch (const std::exception& e) {
        std::cerr << "ERROR: " << e.what() << std::endl;
        return 1;
    }
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::cout << "vacuum lambda:      " << r.lambda << std::endl;
    if (r.alpha != 0.0) {
        std::cout << "focusing angle:     " << r.alpha << " (" << std::sin(r.alpha) * n[0] << " NA)" << std::endl;
        if (r.beta > 0.0)
            std::cout << "obscuration angle:  " << r.beta << " (" << std::sin(r.beta) * n[0] << " NA)" << std::endl;
    }
    std::cout << "layers: " << L << ", incident waves: " << cw.Pi.size() << std::endl;
    std::cout << "output file: " << out << " (" << secs << " s)" << std::endl;
    return 0;
}
