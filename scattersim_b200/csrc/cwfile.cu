// Streaming .cw writer: a CoupledWaveStructure file (CoupledWaveStructure.h:
// 63-125) written straight from a device wave table.
//
// Layout: u64 sizeof(double) = 8; u64 #Pi, the Pi records; u64 #layers; per
// layer: double z, u64 #Pr, records, u64 #Pt, records.  A record is 80 bytes,
// {E0 pair, kx, ky, kz} as complex128.  The E0 pair is stored in the record
// frame of tira::planewave (the frame rotated from z-hat to Re k / |Re k| by
// the minimal rotation; straight-down waves take a half turn about x), or as
// the Cartesian (E_x, E_y) pair.  The wave table's order (Pi, then per
// boundary its Pr and its Pt list) is the file's order, so the file is the
// records of the table with the count fields between the lists.
//
// Records are formed on the device (one thread per wave, the frame arithmetic
// of the host writer term by term with explicitly rounded operations so that
// the bytes agree with it), in chunks of CW_CHUNK records that go through two
// pinned host buffers: chunk c+1 is formed and copied while chunk c is written,
// so a multi-GB file costs about the disk time.
#include <cmath>
#include <cstdio>
#include <vector>

#include "common.cuh"
#include "context.cuh"
#include "kernels.cuh"

namespace sc {

namespace {

constexpr long long CW_CHUNK = 1 << 20;   // records per chunk (80 MB)

// the record pair of one wave: tira frame (frame 0), Cartesian (frame 1), or
// tira frame with a downward wave (Re k_z < 0) in the frame of its z-mirrored
// direction (frame 2: the reference's constructor-made reflected waves)
__global__ void cw_record_kernel(const double2* __restrict__ E0, const double2* __restrict__ K, long long w0,
                                 long long count, int frame, double2* __restrict__ rec) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const long long w = w0 + t;
    const double2 e0 = E0[w * 3], e1 = E0[w * 3 + 1], e2 = E0[w * 3 + 2];
    const double2 k0 = K[w * 3], k1 = K[w * 3 + 1], k2 = K[w * 3 + 2];
    double2 p0, p1;
    if (frame == 1) {
        p0 = e0;
        p1 = e1;
    } else {
        // R with third column Re k / |Re k| (record_frame of the host writer)
        double kh0 = k0.x, kh1 = k1.x, kh2 = (frame == 2) ? fabs(k2.x) : k2.x;
        const double nk = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(kh0, kh0), __dmul_rn(kh1, kh1)),
                                               __dmul_rn(kh2, kh2)));
        kh0 = nk > 0 ? __ddiv_rn(kh0, nk) : 0.0;
        kh1 = nk > 0 ? __ddiv_rn(kh1, nk) : 0.0;
        kh2 = nk > 0 ? __ddiv_rn(kh2, nk) : 0.0;
        const double ax0 = -kh1, ax1 = kh0;
        const double s2 = __dadd_rn(__dmul_rn(ax0, ax0), __dmul_rn(ax1, ax1));
        double R00, R01, R10, R11, R20, R21;
        if (s2 < 1e-30) {
            const double sg = kh2 >= 0 ? 1.0 : -1.0;
            R00 = 1.0;
            R01 = 0.0;
            R10 = 0.0;
            R11 = sg;
            R20 = 0.0;
            R21 = 0.0;
        } else {
            const double f = __ddiv_rn(__dsub_rn(1.0, kh2), s2);
            R00 = __dsub_rn(1.0, __dmul_rn(__dmul_rn(f, ax1), ax1));
            R01 = __dmul_rn(__dmul_rn(f, ax0), ax1);
            R10 = R01;
            R11 = __dsub_rn(1.0, __dmul_rn(__dmul_rn(f, ax0), ax0));
            R20 = -ax1;
            R21 = ax0;
        }
        // out[c] = R[0][c] E_x + R[1][c] E_y + R[2][c] E_z, each a real x complex product
        auto comb = [](double a, double b, double c, double2 x, double2 y, double2 z) {
            return make_double2(__dadd_rn(__dadd_rn(__dmul_rn(a, x.x), __dmul_rn(b, y.x)), __dmul_rn(c, z.x)),
                                __dadd_rn(__dadd_rn(__dmul_rn(a, x.y), __dmul_rn(b, y.y)), __dmul_rn(c, z.y)));
        };
        p0 = comb(R00, R10, R20, e0, e1, e2);
        p1 = comb(R01, R11, R21, e0, e1, e2);
    }
    double2* r = rec + t * 5;
    r[0] = p0;
    r[1] = p1;
    r[2] = k0;
    r[3] = k1;
    r[4] = k2;
}

}  // namespace

sc_status cw_write(sc_context* ctx, const char* path, const double2* E0, const double2* K, long long nw, int layers,
                   const double* z_layers, const long long* counts, int frame, cudaStream_t st) {
    long long total = counts[0];
    for (int l = 0; l < layers; ++l) total += counts[1 + 2 * l] + counts[2 + 2 * l];
    if (total != nw) {
        set_error("sc_cw_write: the list counts add up to %lld, the table holds %lld waves", total, nw);
        return SC_BADINPUT;
    }
    FILE* f = std::fopen(path, "wb");
    if (!f) {
        set_error("sc_cw_write: cannot create %s", path);
        return SC_BADINPUT;
    }
    // the file as a sequence of pieces: header bytes, or a record range [w0, w1)
    struct Piece {
        std::vector<unsigned char> bytes;
        long long w0 = 0, w1 = 0;
    };
    std::vector<Piece> pieces;
    auto put = [&](const void* p, size_t n) {
        if (pieces.empty() || pieces.back().w1 > pieces.back().w0) pieces.push_back(Piece());
        const unsigned char* c = static_cast<const unsigned char*>(p);
        pieces.back().bytes.insert(pieces.back().bytes.end(), c, c + n);
    };
    auto recs = [&](long long w0, long long n) {
        for (long long a = w0; a < w0 + n; a += CW_CHUNK) {
            Piece pc;
            pc.w0 = a;
            pc.w1 = std::min(w0 + n, a + CW_CHUNK);
            pieces.push_back(pc);
        }
    };
    const uint64_t sz = 8;
    put(&sz, 8);
    uint64_t v = (uint64_t)counts[0];
    put(&v, 8);
    recs(0, counts[0]);
    const uint64_t nl = (uint64_t)layers;
    put(&nl, 8);
    long long pos = counts[0];
    for (int l = 0; l < layers; ++l) {
        put(&z_layers[l], 8);
        v = (uint64_t)counts[1 + 2 * l];
        put(&v, 8);
        recs(pos, counts[1 + 2 * l]);
        pos += counts[1 + 2 * l];
        v = (uint64_t)counts[2 + 2 * l];
        put(&v, 8);
        recs(pos, counts[2 + 2 * l]);
        pos += counts[2 + 2 * l];
    }
    double2* dstage;
    sc_status s = ctx->ws.get(&dstage, (size_t)2 * CW_CHUNK * 5, WS_CW_STAGE, st);
    if (s != SC_OK) {
        std::fclose(f);
        return s;
    }
    const long long chunk_recs = std::min(CW_CHUNK, std::max(nw, 1LL));
    double2* host[2] = {nullptr, nullptr};
    cudaEvent_t ev[2] = {nullptr, nullptr};
    sc_status rc = SC_OK;
    for (int i = 0; i < 2 && rc == SC_OK; ++i) {
        if (cudaHostAlloc(&host[i], sizeof(double2) * 5 * chunk_recs, cudaHostAllocDefault) != cudaSuccess ||
            cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            set_error("sc_cw_write: pinned staging allocation failed");
            rc = SC_OOM;
        }
    }
    // record chunks are launched one ahead of the file writes
    int slot_of_prev = -1;
    const Piece* prev = nullptr;
    int slot = 0;
    auto flush_prev = [&]() -> bool {
        if (!prev) return true;
        if (cudaEventSynchronize(ev[slot_of_prev]) != cudaSuccess) return false;
        const size_t nb = (size_t)(prev->w1 - prev->w0) * 80;
        return std::fwrite(host[slot_of_prev], 1, nb, f) == nb;
    };
    for (size_t i = 0; i < pieces.size() && rc == SC_OK; ++i) {
        const Piece& pc = pieces[i];
        if (pc.w1 == pc.w0) {
            // header bytes: everything before them must be on disk first
            if (!flush_prev()) rc = SC_CUDA_ERROR;
            prev = nullptr;
            if (rc == SC_OK && std::fwrite(pc.bytes.data(), 1, pc.bytes.size(), f) != pc.bytes.size()) rc = SC_BADINPUT;
            continue;
        }
        const long long n = pc.w1 - pc.w0;
        double2* dd = dstage + (size_t)slot * CW_CHUNK * 5;
        cw_record_kernel<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(E0, K, pc.w0, n, frame, dd);
        count_launch();
        if (cudaGetLastError() != cudaSuccess ||
            cudaMemcpyAsync(host[slot], dd, sizeof(double2) * 5 * n, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaEventRecord(ev[slot], st) != cudaSuccess) {
            rc = SC_CUDA_ERROR;
            break;
        }
        if (!flush_prev()) {
            rc = SC_CUDA_ERROR;
            break;
        }
        prev = &pc;
        slot_of_prev = slot;
        slot ^= 1;
    }
    if (rc == SC_OK && !flush_prev()) rc = SC_CUDA_ERROR;
    cudaStreamSynchronize(st);
    for (int i = 0; i < 2; ++i) {
        if (host[i]) cudaFreeHost(host[i]);
        if (ev[i]) cudaEventDestroy(ev[i]);
    }
    if (std::fclose(f) != 0 && rc == SC_OK) rc = SC_BADINPUT;
    if (rc == SC_CUDA_ERROR) set_error("sc_cw_write: a record copy or the write to %s failed", path);
    else if (rc == SC_BADINPUT) set_error("sc_cw_write: writing %s failed", path);
    return rc;
}

}  // namespace sc
