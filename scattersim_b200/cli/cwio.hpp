// Host-side I/O for the command-line tools: long-option parsing in the style
// of the reference's boost::program_options setup (ScatterVolume.cpp:510-536:
// long options only, multi-token values, negative numbers allowed), .npy
// read/write, and the coupled-wave (.cw) file of CoupledWaveStructure.h:63-125.
#pragma once

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
struct Wave {
    cplx E[3];
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

inline void put_records(std::ofstream& f, const std::vector<Wave>& w) {
    uint64_t n = w.size();
    f.write((const char*)&n, 8);
    for (auto& x : w) {
        cplx rec[5] = {x.E[0], x.E[1], x.k[0], x.k[1], x.k[2]};
        f.write((const char*)rec, sizeof(rec));
    }
}

inline void save_cw(const std::string& path, const CoupledWave& cw) {
    std::ofstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("cannot write " + path);
    uint64_t sz = 8;
    f.write((const char*)&sz, 8);
    put_records(f, cw.Pi);
    uint64_t nl = cw.layers.size();
    f.write((const char*)&nl, 8);
    for (auto& L : cw.layers) {
        f.write((const char*)&L.z, 8);
        put_records(f, L.Pr);
        put_records(f, L.Pt);
    }
}

inline std::vector<Wave> get_records(std::ifstream& f) {
    uint64_t n = 0;
    f.read((char*)&n, 8);
    std::vector<Wave> w(n);
    for (auto& x : w) {
        cplx rec[5];
        f.read((char*)rec, sizeof(rec));
        x.E[0] = rec[0];
        x.E[1] = rec[1];
        x.k[0] = rec[2];
        x.k[1] = rec[3];
        x.k[2] = rec[4];
        // E_z by transversality (k . E = 0)
        x.E[2] = (x.k[2] == cplx(0.0)) ? cplx(0.0) : -(x.k[0] * x.E[0] + x.k[1] * x.E[1]) / x.k[2];
    }
    return w;
}

inline CoupledWave load_cw(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) throw std::runtime_error("file " + path + " not found");
    uint64_t sz = 0;
    f.read((char*)&sz, 8);
    if (sz != 8) throw std::runtime_error(path + ": only double-precision .cw files are supported");
    CoupledWave cw;
    cw.Pi = get_records(f);
    uint64_t nl = 0;
    f.read((char*)&nl, 8);
    cw.layers.resize(nl);
    for (auto& L : cw.layers) {
        f.read((char*)&L.z, 8);
        L.Pr = get_records(f);
        L.Pt = get_records(f);
    }
    if (!f) throw std::runtime_error(path + ": truncated");
    return cw;
}

}  // namespace cwio
