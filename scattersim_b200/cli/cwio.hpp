// Host-side I/O for the command-line tools: long-option parsing in the style
// of the reference's boost::program_options setup (ScatterVolume.cpp:510-536:
// long options only, multi-token values, negative numbers allowed), .npy
// read/write, and the coupled-wave (.cw) file of CoupledWaveStructure.h:63-125.
#pragma once

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <stdexcept>
#include <string>
#include <vector>

namespace cwio {

using cplx = std::complex<double>;

// ------------------------------------------------------------------ options
struct Options {
    std::map<std::string, std::vector<std::string>> values;
    bool has(const std::string& k) const { return values.count(k) != 0; }
    std::vector<double> nums(const std::string& k, std::vector<double> dflt) const {
        auto it = values.find(k);
        if (it == values.end()) return dflt;
        std::vector<double> out;
        for (auto& s : it->second) out.push_back(std::strtod(s.c_str(), nullptr));
        return out;
    }
    double num(const std::string& k, double dflt) const {
        auto v = nums(k, {dflt});
        return v.empty() ? dflt : v[0];
    }
    std::string str(const std::string& k, const std::string& dflt) const {
        auto it = values.find(k);
        return (it == values.end() || it->second.empty()) ? dflt : it->second[0];
    }
};

inline bool is_option(const char* a) {
    if (std::strncmp(a, "--", 2) != 0) return false;
    // "--" followed by a digit or '.' is a negative number, not an option
    return !(a[2] >= '0' && a[2] <= '9') && a[2] != '.';
}

inline Options parse(int argc, char** argv, const std::vector<std::string>& known,
                     const std::string& positional = "") {
    Options o;
    std::string cur;
    for (int i = 1; i < argc; ++i) {
        if (is_option(argv[i])) {
            cur = argv[i] + 2;
            bool ok = false;
            for (auto& k : known) ok = ok || (k == cur);
            if (!ok) throw std::runtime_error("unrecognised option '--" + cur + "'");
            o.values[cur];
        } else if (!cur.empty()) {
            o.values[cur].push_back(argv[i]);
        } else if (!positional.empty()) {
            o.values[positional].push_back(argv[i]);
        } else {
            throw std::runtime_error(std::string("unexpected argument '") + argv[i] + "'");
        }
    }
    return o;
}

// ------------------------------------------------------------------ .npy
struct NpyArray {
    std::vector<size_t> shape;
    std::string descr;
    std::vector<char> data;
};

inline NpyArray read_npy(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot open " + path);
    char magic[6];
    f.read(magic, 6);
    if (std::memcmp(magic, "\x93NUMPY", 6) != 0) throw std::runtime_error(path + ": not an .npy file");
    unsigned char ver[2];
    f.read((char*)ver, 2);
    uint32_t hlen = 0;
    if (ver[0] == 1) {
        uint16_t h16;
        f.read((char*)&h16, 2);
        hlen = h16;
    } else {
        f.read((char*)&hlen, 4);
    }
    std::string hdr(hlen, ' ');
    f.read(&hdr[0], hlen);
    NpyArray a;
    auto d = hdr.find("'descr'");
    auto q1 = hdr.find('\'', d + 7), q2 = hdr.find('\'', hdr.find('\'', d + 7) + 1);
    a.descr = hdr.substr(q1 + 1, q2 - q1 - 1);
    if (hdr.find("'fortran_order': True") != std::string::npos)
        throw std::runtime_error(path + ": Fortran-ordered arrays are not supported");
    auto s0 = hdr.find('(', hdr.find("'shape'")), s1 = hdr.find(')', s0);
    std::string sh = hdr.substr(s0 + 1, s1 - s0 - 1);
    size_t pos = 0;
    while (pos < sh.size()) {
        while (pos < sh.size() && (sh[pos] == ' ' || sh[pos] == ',')) ++pos;
        if (pos >= sh.size()) break;
        a.shape.push_back(std::strtoull(sh.c_str() + pos, nullptr, 10));
        while (pos < sh.size() && sh[pos] != ',') ++pos;
    }
    size_t count = 1;
    for (auto s : a.shape) count *= s;
    size_t item = (a.descr == "<c16") ? 16 : (a.descr == "<c8") ? 8 : (a.descr == "<f8") ? 8 : 0;
    if (!item) throw std::runtime_error(path + ": unsupported dtype " + a.descr);
    a.data.resize(count * item);
    f.read(a.data.data(), (std::streamsize)a.data.size());
    if ((size_t)f.gcount() != a.data.size()) throw std::runtime_error(path + ": truncated");
    return a;
}

inline void write_npy(const std::string& path, const std::string& descr, const std::vector<size_t>& shape,
                      const void* data, size_t bytes) {
    std::string sh = "(";
    for (size_t i = 0; i < shape.size(); ++i) sh += std::to_string(shape[i]) + (shape.size() == 1 ? "," : (i + 1 < shape.size() ? ", " : ""));
    sh += ")";
    std::string hdr = "{'descr': '" + descr + "', 'fortran_order': False, 'shape': " + sh + ", }";
    size_t total = 10 + hdr.size() + 1;
    hdr += std::string((64 - total % 64) % 64, ' ') + "\n";
    std::ofstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot write " + path);
    f.write("\x93NUMPY\x01\x00", 8);
    uint16_t hl = (uint16_t)hdr.size();
    f.write((const char*)&hl, 2);
    f.write(hdr.data(), (std::streamsize)hdr.size());
    f.write((const char*)data, (std::streamsize)bytes);
}

// ------------------------------------------------------------------ .cw
// One record = {E0x, E0y, kx, ky, kz} complex128 (80 bytes); E0z is not stored.
//
// Record frame (Frame::tira, the default): tira's planewave keeps E0 in a
// frame whose z axis is the real propagation direction Re(k)/|Re(k)| (the
// minimal rotation taking z-hat there) and the file holds the first two
// components in that frame; the reader rebuilds the third from k . E = 0 in
// the same frame.  This is the reading under which every record of the
// reference's data/psf.cw, and the incident and transmitted records of
// x64/a.cw, equal the restated solves of their runs.  Frame::tira_mirror
// ('tira-mirror') takes, for a downward wave (Re k_z < 0), the frame of the
// z-mirrored direction (Re k_x, Re k_y, -Re k_z): the frame in which the
// reference's scatterlayer stores its reflected waves (made by tira's
// planewave constructor, ScatterLayer.cpp:246-251), under which every record
// of x64/a.cw equals the restated solve; scatterplane's waves (made by tira's
// scatter(), ScatterPlane.cpp:175, 244) keep their own frame (Frame::tira).
// Frame::cartesian stores (E_x, E_y) and rebuilds E_z from k . E = 0 (not
// the reference's convention; kept for files written that way).
struct Wave {
    cplx E[3];   // Cartesian E0
    cplx k[3];
};
struct Boundary {
    double z = 0.0;
    std::vector<Wave> Pr, Pt;
};
struct CoupledWave {
    std::vector<Wave> Pi;
    std::vector<Boundary> layers;
};

// Frame::automatic is for readers only: the file's own convention, decided
// from the field's continuity at its first interface (load_cw).
enum class Frame { tira, tira_mirror, cartesian, automatic };

inline Frame parse_frame(const std::string& s) {
    if (s == "tira") return Frame::tira;
    if (s == "tira-mirror") return Frame::tira_mirror;
    if (s == "cartesian") return Frame::cartesian;
    throw std::runtime_error("unknown --cw-frame '" + s + "' (tira, tira-mirror or cartesian)");
}
inline Frame parse_read_frame(const std::string& s) {
    if (s == "auto") return Frame::automatic;
    if (s == "tira" || s == "tira-mirror" || s == "cartesian") return parse_frame(s);
    throw std::runtime_error("unknown --cw-frame '" + s + "' (tira, tira-mirror, cartesian or auto)");
}

// R (row-major) with third column Re(k)/|Re(k)|: minimal rotation from z-hat;
// straight down is a half turn about x.  mirror_down: a downward wave takes
// the rotation of its z-mirrored direction.
inline void record_frame(const cplx k[3], double R[3][3], bool mirror_down = false) {
    double kh[3] = {k[0].real(), k[1].real(), mirror_down ? std::fabs(k[2].real()) : k[2].real()};
    const double nk = std::sqrt(kh[0] * kh[0] + kh[1] * kh[1] + kh[2] * kh[2]);
    for (double& v : kh) v = nk > 0 ? v / nk : 0.0;
    const double ax0 = -kh[1], ax1 = kh[0], s2 = ax0 * ax0 + ax1 * ax1;
    if (s2 < 1e-30) {
        const double sg = kh[2] >= 0 ? 1.0 : -1.0;
        const double I[3][3] = {{1, 0, 0}, {0, sg, 0}, {0, 0, sg}};
        std::memcpy(R, I, sizeof(I));
        return;
    }
    const double f = (1.0 - kh[2]) / s2;
    const double M[3][3] = {{1.0 - f * ax1 * ax1, f * ax0 * ax1, ax1},
                            {f * ax0 * ax1, 1.0 - f * ax0 * ax0, -ax0},
                            {-ax1, ax0, kh[2]}};
    std::memcpy(R, M, sizeof(M));
}

inline void to_record(const Wave& w, Frame fr, cplx out[2]) {
    if (fr == Frame::automatic) throw std::runtime_error("a .cw file is written in one named record frame");
    if (fr == Frame::cartesian) {
        out[0] = w.E[0];
        out[1] = w.E[1];
        return;
    }
    double R[3][3];
    record_frame(w.k, R, fr == Frame::tira_mirror);
    for (int c = 0; c < 2; ++c) out[c] = R[0][c] * w.E[0] + R[1][c] * w.E[1] + R[2][c] * w.E[2];
}

inline void from_record(const cplx p[2], Wave& w, Frame fr) {
    if (fr == Frame::cartesian) {
        w.E[0] = p[0];
        w.E[1] = p[1];
        w.E[2] = (w.k[2] == cplx(0.0)) ? cplx(0.0) : -(w.k[0] * p[0] + w.k[1] * p[1]) / w.k[2];
        return;
    }
    double R[3][3];
    record_frame(w.k, R, fr == Frame::tira_mirror);
    cplx kp[3];
    for (int c = 0; c < 3; ++c) kp[c] = R[0][c] * w.k[0] + R[1][c] * w.k[1] + R[2][c] * w.k[2];
    const cplx e2 = (kp[2] == cplx(0.0)) ? cplx(0.0) : -(kp[0] * p[0] + kp[1] * p[1]) / kp[2];
    for (int r = 0; r < 3; ++r) w.E[r] = R[r][0] * p[0] + R[r][1] * p[1] + R[r][2] * e2;
}

inline void put_records(std::ofstream& f, const std::vector<Wave>& w, Frame fr) {
    uint64_t n = w.size();
    f.write((const char*)&n, 8);
    for (auto& x : w) {
        cplx rec[5];
        to_record(x, fr, rec);
        rec[2] = x.k[0];
        rec[3] = x.k[1];
        rec[4] = x.k[2];
        f.write((const char*)rec, sizeof(rec));
    }
}

inline void save_cw(const std::string& path, const CoupledWave& cw, Frame fr = Frame::tira) {
    std::ofstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot write " + path);
    uint64_t sz = 8;
    f.write((const char*)&sz, 8);
    put_records(f, cw.Pi, fr);
    uint64_t nl = cw.layers.size();
    f.write((const char*)&nl, 8);
    for (auto& L : cw.layers) {
        f.write((const char*)&L.z, 8);
        put_records(f, L.Pr, fr);
        put_records(f, L.Pt, fr);
    }
}

inline std::vector<Wave> get_records(std::ifstream& f, Frame fr) {
    uint64_t n = 0;
    f.read((char*)&n, 8);
    if (!f || n > (uint64_t(1) << 40)) throw std::runtime_error("corrupt record count");
    std::vector<Wave> w(n);
    for (auto& x : w) {
        cplx rec[5];
        f.read((char*)rec, sizeof(rec));
        x.k[0] = rec[2];
        x.k[1] = rec[3];
        x.k[2] = rec[4];
        from_record(rec, x, fr);
    }
    return w;
}

// Largest jump of the tangential (x, y) field across the first interface,
// relative to the field there, with the stored pairs (held in E[0], E[1] of
// `raw`) read in frame fr: the plane-wave sum of region 0 (incident +
// reflected at z_0) against region 1 (transmitted at z_0 + reflected at z_1),
// on the plane z = z_0 at eight points within a wavelength of the axis (the
// regions of cpuEvaluator.cpp:34-102).  The reading a file was written in
// gives a continuous field.
inline double interface_jump(const CoupledWave& raw, Frame fr) {
    if (raw.layers.empty()) return 0.0;
    const Boundary& L0 = raw.layers[0];
    std::vector<const std::vector<Wave>*> above = {&raw.Pi, &L0.Pr}, below = {&L0.Pt};
    if (raw.layers.size() > 1) below.push_back(&raw.layers[1].Pr);
    double kmax = 1.0;
    for (auto* ws : {&raw.Pi, &L0.Pr, &L0.Pt})
        for (auto& w : *ws) kmax = std::max(kmax, std::abs(w.k[0]) + std::abs(w.k[1]) + std::abs(w.k[2]));
    const double off[8][2] = {{0.13, -0.71}, {-0.52, 0.38}, {0.91, 0.07}, {-0.26, -0.44},
                              {0.47, 0.83}, {-0.88, -0.19}, {0.05, 0.56}, {0.64, -0.33}};
    const double wl = 2.0 * M_PI / kmax;
    double jump = 0.0, scale = 0.0;
    for (auto& o : off) {
        const double r[3] = {o[0] * wl, o[1] * wl, L0.z};
        cplx Ea[2] = {0.0, 0.0}, Eb[2] = {0.0, 0.0};
        auto add = [&](const std::vector<const std::vector<Wave>*>& lists, cplx E[2]) {
            for (auto* ws : lists)
                for (const Wave& w0 : *ws) {
                    Wave w = w0;
                    const cplx p[2] = {w0.E[0], w0.E[1]};
                    from_record(p, w, fr);
                    const cplx ph = std::exp(cplx(0.0, 1.0) * (w.k[0] * r[0] + w.k[1] * r[1] + w.k[2] * r[2]));
                    E[0] += w.E[0] * ph;
                    E[1] += w.E[1] * ph;
                }
        };
        add(above, Ea);
        add(below, Eb);
        for (int c = 0; c < 2; ++c) {
            jump = std::max(jump, std::abs(Ea[c] - Eb[c]));
            scale = std::max(scale, std::max(std::abs(Ea[c]), std::abs(Eb[c])));
        }
    }
    return scale > 0.0 ? jump / scale : 0.0;
}

inline CoupledWave load_cw(const std::string& path, Frame fr = Frame::tira) {
    if (fr == Frame::automatic) {
        CoupledWave cw = load_cw(path, Frame::cartesian);     // E[0], E[1]: the stored pairs
        const Frame use = interface_jump(cw, Frame::tira_mirror) < interface_jump(cw, Frame::tira)
                              ? Frame::tira_mirror : Frame::tira;
        auto conv = [&](std::vector<Wave>& ws) {
            for (Wave& w : ws) {
                const cplx p[2] = {w.E[0], w.E[1]};
                from_record(p, w, use);
            }
        };
        conv(cw.Pi);
        for (auto& L : cw.layers) {
            conv(L.Pr);
            conv(L.Pt);
        }
        return cw;
    }
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("file " + path + " not found");
    uint64_t sz = 0;
    f.read((char*)&sz, 8);
    if (sz != 8) throw std::runtime_error(path + ": only double-precision .cw files are supported");
    CoupledWave cw;
    cw.Pi = get_records(f, fr);
    uint64_t nl = 0;
    f.read((char*)&nl, 8);
    if (!f || nl > (uint64_t(1) << 20)) throw std::runtime_error(path + ": corrupt layer count");
    cw.layers.resize(nl);
    for (auto& L : cw.layers) {
        f.read((char*)&L.z, 8);
        L.Pr = get_records(f, fr);
        L.Pt = get_records(f, fr);
    }
    if (!f) throw std::runtime_error(path + ": truncated");
    return cw;
}

}  // namespace cwio
