// scatterplane: the reference's single-interface program over the C ABI.
//
// Same long options and defaults as ScatterPlane.cpp:85-103 (--lambda,
// --direction, --focus, --ex, --ey, --ez, --n, --kappa, --z, --output,
// --alpha, --beta, --samples, --mode, --wavemask, --log, --nooutput).  The
// focused beam (polar mode, :154-171, 236-242) is wound to the focal point and
// every wave is refracted at the plane z between n[0] and n[1] + i kappa
// (:175, 243-256) -- the two-layer case of the batched layer solve, which
// reproduces the reference's shipped data/psf.cw to rounding.  The .cw layout
// is the reference's (records in its record frame).  --mode montecarlo is
// refused: its random sampler (tira) is not available.
#include <chrono>
#include <cmath>
#include <iostream>

#include "layercli.hpp"

int main(int argc, char** argv) {
    const std::vector<std::string> known = {"help", "lambda", "direction", "focus", "ex", "ey", "ez", "n", "kappa",
                                            "z", "output", "alpha", "beta", "samples", "mode", "wavemask", "log",
                                            "nooutput", "cuda", "cw-frame"};
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
                     "  --direction arg (=1, 0, 1) incoming field direction\n"
                     "  --focus arg (=0, 0, 0) focal point for the incident field\n"
                     "  --ex arg (=0 0)        x component of the electrical field\n"
                     "  --ey arg (=1 0)        y component of the electrical field\n"
                     "  --ez arg (=0 0)        z component of the electrical field\n"
                     "  --n arg (=1.0 1.4)     layer refractive indices\n"
                     "  --kappa arg (=0.05)    transmitted material absorption coefficient\n"
                     "  --z arg (=0)           position of the plane along the z axis\n"
                     "  --output arg (=a.cw)   output filename for the coupled wave structure\n"
                     "  --alpha arg (=0.5)     angle used to focus the incident field\n"
                     "  --beta arg (=0)        internal obscuration angle (for simulating reflective optics)\n"
                     "  --samples arg (=375)   number of samples (can be specified in 2 dimensions)\n"
                     "  --mode arg (=polar)    sampling mode (polar)\n"
                     "  --wavemask arg (=1 1 1) waves simulated (boolean value for incident, reflected, and "
                     "transmitted)\n"
                     "  --nooutput             save an output file without printing the summary\n"
                     "  --cw-frame arg (=tira) record frame of the written .cw ('tira', 'tira-mirror' or 'cartesian')\n";
        return 1;
    }
    auto t0 = std::chrono::steady_clock::now();
    layercli::Run r;
    r.lambda = o.num("lambda", 1.0);
    auto dir = o.nums("direction", {1, 0, 1}), foc = o.nums("focus", {0, 0, 0});
    auto ex = o.nums("ex", {0, 0}), ey = o.nums("ey", {1, 0}), ez = o.nums("ez", {0, 0});
    auto n = o.nums("n", {1.0, 1.4});
    auto mask = o.nums("wavemask", {1, 1, 1});
    if (dir.size() < 3 || foc.size() < 3 || ex.size() < 2 || ey.size() < 2 || ez.size() < 2 || n.size() < 2 ||
        mask.size() < 3) {
        std::cerr << "ERROR: --direction/--focus/--wavemask take 3 values, --ex/--ey/--ez/--n 2" << std::endl;
        return 1;
    }
    for (int i = 0; i < 3; ++i) {
        r.dir[i] = dir[i];
        r.focus[i] = foc[i];
        r.wave_mask[i] = mask[i] != 0.0;
    }
    r.e[0] = {ex[0], ex[1]};
    r.e[1] = {ey[0], ey[1]};
    r.e[2] = {ez[0], ez[1]};
    r.n = {n[0], n[1]};
    r.kappa = {o.num("kappa", 0.05)};
    r.z = {o.num("z", 0.0)};
    r.alpha = o.num("alpha", 0.5);
    r.beta = o.num("beta", 0.0);
    layercli::samples(o.nums("samples", {64, 64}), r.N0, r.N1);
    if (o.str("mode", "polar") != "polar") {
        std::cerr << "ERROR: only --mode polar is supported (the Monte Carlo sampler's generator is not available)"
                  << std::endl;
        return 1;
    }
    if (r.alpha == 0.0) r.N0 = r.N1 = 1;                                      // :168-171
    r.device = (int)o.num("cuda", 0);
    cwio::Frame frame;
    try {
        frame = cwio::parse_frame(o.str("cw-frame", "tira"));
    } catch (const std::exception& e) {
        std::cerr << "ERROR: " << e.what() << std::endl;
        return 1;
    }
    if (r.N0 * r.N1 == 1)                                                     // :215-218 write all three lists
        for (int i = 0; i < 3; ++i) r.wave_mask[i] = true;
    cwio::CoupledWave cw;
    if (layercli::solve(r, cw)) return 1;
    const std::string out = o.str("output", "a.cw");
    try {
        if (!out.empty()) cwio::save_cw(out, cw, frame);
    } catch (const std::exception& e) {
        std::cerr << "ERROR: " << e.what() << std::endl;
        return 1;
    }
    if (!o.has("nooutput")) {
        const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        std::cout << "vacuum wavelength:            " << r.lambda << std::endl;
        std::cout << "focal point:                  " << r.focus[0] << " " << r.focus[1] << " " << r.focus[2]
                  << std::endl;
        if (r.alpha != 0.0) {
            std::cout << "focusing angle:               " << r.alpha << " (" << std::sin(r.alpha) * n[0] << " NA)"
                      << std::endl;
            if (r.beta > 0.0)
                std::cout << "obscuration angle:            " << r.beta << " (" << std::sin(r.beta) * n[0]
                          << " NA)" << std::endl;
        }
        std::cout << "samples:                      " << r.N0 << " x " << r.N1 << " = " << r.N0 * r.N1 << std::endl;
        std::cout << "sampling mode:                polar" << std::endl;
        std::cout << "output file:                  " << out << " (" << secs << " s)" << std::endl;
    }
    return 0;
}
