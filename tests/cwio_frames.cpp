// Test harness for the command-line tools' .cw record frames (cli/cwio.hpp),
// built and run on the CPU by tests/test_cwfile.py:
//   cwio_frames <in.cw> <frame> <out.cw> <fields.bin>
// loads <in.cw> reading its records in <frame> (tira, tira-mirror,
// cartesian, or auto: decided from the field's continuity at the first
// interface), writes the Cartesian E0 of every wave (incident, then per
// boundary reflected and transmitted; 3 complex128 each) to <fields.bin> and,
// for a named frame, saves the waves again to <out.cw> in that frame.
#include "cwio.hpp"

int main(int argc, char** argv) {
    if (argc != 5) {
        std::fprintf(stderr, "usage: cwio_frames in.cw frame out.cw fields.bin\n");
        return 2;
    }
    try {
        const cwio::Frame fr = cwio::parse_read_frame(argv[2]);
        const cwio::CoupledWave cw = cwio::load_cw(argv[1], fr);
        std::ofstream f(argv[4], std::ios::binary);
        auto dump = [&](const std::vector<cwio::Wave>& w) {
            for (auto& x : w) f.write((const char*)x.E, sizeof(x.E));
        };
        dump(cw.Pi);
        for (auto& L : cw.layers) {
            dump(L.Pr);
            dump(L.Pt);
        }
        if (fr != cwio::Frame::automatic) cwio::save_cw(argv[3], cw, fr);
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ERROR: %s\n", e.what());
        return 1;
    }
    return 0;
}
