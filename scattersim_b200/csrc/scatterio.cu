// ScatterIO files: single scattering events at one boundary plane.
//
// The reference's ScatterIO.h (write_file :18-42, read_file :44-87 and the
// single-beam / single-event overloads :89-117) stores, in native byte order:
//   the plane normal and a point on the plane   2 x 3 doubles
//   per beam: N (size_t), then N triples of     8 bytes
//     incident, reflected, transmitted records  3 x 80 bytes
// A record is a tira planewave<double>: {E0x, E0y, kx, ky, kz} as complex128
// (the 80-byte record of the .cw file).  The reader takes beams until a count
// is zero or missing (end of file).  Host code only: these are file formats,
// not device work.
#include <cstdio>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace {
constexpr size_t SIO_RECORD = 80;
}

extern "C" {

sc_status sc_scatterio_write(const char* path, const double* normal, const double* position, int beams,
                             const long long* counts, const void* incident, const void* reflected,
                             const void* transmitted) {
    if (!path || !normal || !position || beams < 0 || (beams > 0 && !counts)) {
        sc::set_error("sc_scatterio_write: bad argument");
        return SC_BADINPUT;
    }
    long long total = 0;
    for (int b = 0; b < beams; ++b) {
        if (counts[b] < 0) {
            sc::set_error("sc_scatterio_write: beam %d has a negative count", b);
            return SC_BADINPUT;
        }
        total += counts[b];
    }
    if (total > 0 && (!incident || !reflected || !transmitted)) {
        sc::set_error("sc_scatterio_write: null record array");
        return SC_BADINPUT;
    }
    FILE* f = std::fopen(path, "wb");
    if (!f) {
        sc::set_error("sc_scatterio_write: cannot create %s", path);
        return SC_BADINPUT;
    }
    bool ok = std::fwrite(normal, sizeof(double), 3, f) == 3 && std::fwrite(position, sizeof(double), 3, f) == 3;
    const unsigned char* pi = static_cast<const unsigned char*>(incident);
    const unsigned char* pr = static_cast<const unsigned char*>(reflected);
    const unsigned char* pt = static_cast<const unsigned char*>(transmitted);
    long long off = 0;
    for (int b = 0; b < beams && ok; ++b) {
        const size_t N = (size_t)counts[b];
        ok = std::fwrite(&N, sizeof(size_t), 1, f) == 1;
        for (size_t n = 0; n < N && ok; ++n, ++off) {
            ok = std::fwrite(pi + off * SIO_RECORD, 1, SIO_RECORD, f) == SIO_RECORD &&
                 std::fwrite(pr + off * SIO_RECORD, 1, SIO_RECORD, f) == SIO_RECORD &&
                 std::fwrite(pt + off * SIO_RECORD, 1, SIO_RECORD, f) == SIO_RECORD;
        }
    }
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) {
        sc::set_error("sc_scatterio_write: write to %s failed", path);
        return SC_BADINPUT;
    }
    return SC_OK;
}

sc_status sc_scatterio_read(const char* path, double* normal, double* position, int* beams, long long* counts,
                            int beams_cap, void* incident, void* reflected, void* transmitted,
                            long long events_cap, long long* events) {
    if (!path || !normal || !position || !beams || !events || beams_cap < 0 || events_cap < 0) {
        sc::set_error("sc_scatterio_read: bad argument");
        return SC_BADINPUT;
    }
    FILE* f = std::fopen(path, "rb");
    if (!f) {
        sc::set_error("sc_scatterio_read: cannot open %s", path);
        return SC_BADINPUT;
    }
    if (std::fread(normal, sizeof(double), 3, f) != 3 || std::fread(position, sizeof(double), 3, f) != 3) {
        std::fclose(f);
        sc::set_error("sc_scatterio_read: %s is shorter than its plane header", path);
        return SC_BADINPUT;
    }
    unsigned char* pi = static_cast<unsigned char*>(incident);
    unsigned char* pr = static_cast<unsigned char*>(reflected);
    unsigned char* pt = static_cast<unsigned char*>(transmitted);
    const bool copy = pi && pr && pt;
    int nb = 0;
    long long total = 0;
    unsigned char rec[3 * SIO_RECORD];
    while (true) {
        size_t N = 0;
        if (std::fread(&N, sizeof(size_t), 1, f) != 1 || N == 0) break;   // read_file stops here
        if (counts && nb < beams_cap) counts[nb] = (long long)N;
        for (size_t n = 0; n < N; ++n, ++total) {
            if (std::fread(rec, 1, sizeof(rec), f) != sizeof(rec)) {
                std::fclose(f);
                sc::set_error("sc_scatterio_read: %s ends inside beam %d", path, nb);
                return SC_BADINPUT;
            }
            if (copy && total < events_cap) {
                std::memcpy(pi + total * SIO_RECORD, rec, SIO_RECORD);
                std::memcpy(pr + total * SIO_RECORD, rec + SIO_RECORD, SIO_RECORD);
                std::memcpy(pt + total * SIO_RECORD, rec + 2 * SIO_RECORD, SIO_RECORD);
            }
        }
        ++nb;
    }
    std::fclose(f);
    *beams = nb;
    *events = total;
    if ((copy && total > events_cap) || (counts && nb > beams_cap)) {
        sc::set_error("sc_scatterio_read: %s holds %d beams / %lld events, more than the buffers", path, nb, total);
        return SC_BADINPUT;
    }
    return SC_OK;
}

}  // extern "C"
