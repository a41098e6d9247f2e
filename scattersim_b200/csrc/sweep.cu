// Batched sweep of independent scattervolume solves: the R/T amplitude vector
// x = [R; T] of many instances (wavelengths, incidence angles, layer stacks,
// order counts) in one call.  The reference runs one scattervolume process per
// sweep point (videomaker.py:61-74, spectroscopy.py:66-91, with the
// --external solve of ScatterVolume.cpp:739 and no interior fields).
//
// Instances are grouped by their order counts (Mx, My); within a group every
// layer of every instance goes through the same batched kernels:
//   1. fft2_crop per instance into the group's coefficient arrays;
//   2. B, C of every layer (per-layer lattice and k), Omega = B C;
//   3. the inverse layer factors exp(-i k dz Phi) as matrix functions of Omega
//      (mfun.cu), kept in factored form (F, G B, C G) -- no eigendecomposition
//      is needed for R/T;
//   4. the chain X <- T_l^-1 X from f3 up through the stack, four batched
//      GEMMs per depth step over all instances still inside their stack
//      (instances are sorted by depth, so the active ones are a prefix):
//      U = (G B) X2, V = F X1, X1' = F (2 V - t U) - X1,
//      X2' = X2 + (C G) ((t^2/2) U - t V);
//   5. the boundary systems (ScatterVolume.cpp:398-466), batched over
//      instances: the reflected amplitudes enter only through per-order 3 x 3
//      blocks, so they are eliminated order by order and a 3M x 3M system in
//      the transmitted amplitudes is LU-solved (8x fewer flops than the 6M
//      system, which remains the path when an order grazes the top interface).
// A group larger than the memory budget is processed in chunks of instances.
#include <algorithm>
#include <cmath>
#include <map>
#include <utility>

#include "context.cuh"

namespace sc {

namespace {

struct Item {
    int idx = 0;
    VolumePlan plan;
    int Z = 0, S1 = 0, S2 = 0;
    const double2* sample = nullptr;
    double2* x = nullptr;
};

// bump allocator over one device buffer (base == nullptr: measure only)
struct Carve {
    char* base = nullptr;
    size_t off = 0;
    template <typename T>
    T* take(size_t count) {
        const size_t b = (count * sizeof(T) + 255) & ~size_t(255);
        T* p = base ? reinterpret_cast<T*>(base + off) : nullptr;
        off += b;
        return p;
    }
};

// Between the products of one chain step, per instance b (U, V: n2 x ncol, leading
// dimension n2; X: n4 x ncol, leading dimension n4 = 2 n2):
//   V <- 2 V - t U,  U <- (t^2 / 2) U - t V (both from the old U, V),
//   Xn <- Xc (the X1' product then runs with beta = -1, the X2' product with beta = +1)
__global__ void chain_mix_kernel(int n2, int ncol, const double2* __restrict__ tv, double2* const* __restrict__ Up,
                                 double2* const* __restrict__ Vp, const double2* const* __restrict__ Xc,
                                 double2* const* __restrict__ Xn) {
    const int b = blockIdx.y;
    const double2 t = tv[b];
    const double2 t2h = cscale(cmul(t, t), 0.5);
    double2* U = Up[b];
    double2* V = Vp[b];
    const double2* xc = Xc[b];
    double2* xn = Xn[b];
    const long long tot = (long long)n2 * ncol;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < tot;
         e += (long long)gridDim.x * blockDim.x) {
        const int r = (int)(e % n2), c = (int)(e / n2);
        const double2 u = U[e], v = V[e];
        V[e] = csub(cscale(v, 2.0), cmul(t, u));
        U[e] = csub(cmul(t2h, u), cmul(t, v));
        const long long x = (long long)c * (2 * n2) + r;
        xn[x] = xc[x];
        xn[x + n2] = xc[x + n2];
    }
}

struct ChunkBufs {
    double *lat, *kinv, *kz0, *dnorm;
    int *inst, *piv, *info, *bins;
    double2 *svec, *Nf, *Nif, *R2, *Ri2, *B, *C, *Om, *scr, *T, *X0, *X1, *A6, *b6, *coef;
};

ChunkBufs carve_chunk(Carve& cv, int nI, int Ltot, int maxZS1, int Mx, int My) {
    const long long MF = (long long)Mx * My, n2 = 2 * MF, n4 = 4 * MF, n6 = 6 * MF;
    ChunkBufs b;
    b.lat = cv.take<double>((size_t)nI * (Mx + My));
    b.kinv = cv.take<double>(nI);
    b.kz0 = cv.take<double>(2 * (size_t)nI);
    b.dnorm = cv.take<double>(Ltot);
    b.inst = cv.take<int>(Ltot);
    b.piv = cv.take<int>((size_t)nI * n6);
    b.info = cv.take<int>(nI);
    b.bins = cv.take<int>(Mx + My);
    b.svec = cv.take<double2>((size_t)nI * 7 * MF);
    b.Nf = cv.take<double2>((size_t)Ltot * MF);
    b.Nif = cv.take<double2>((size_t)Ltot * MF);
    b.R2 = cv.take<double2>((size_t)maxZS1 * Mx);
    b.Ri2 = cv.take<double2>((size_t)maxZS1 * Mx);
    b.B = cv.take<double2>((size_t)Ltot * n2 * n2);
    b.C = cv.take<double2>((size_t)Ltot * n2 * n2);
    b.Om = cv.take<double2>((size_t)Ltot * n2 * n2);
    b.scr = cv.take<double2>(transfer_scratch_blocks() * Ltot * n2 * n2);
    b.T = cv.take<double2>((size_t)Ltot * n4 * n4);
    b.X0 = cv.take<double2>((size_t)nI * n4 * 3 * MF);
    b.X1 = cv.take<double2>((size_t)nI * n4 * 3 * MF);
    b.A6 = cv.take<double2>((size_t)nI * n6 * n6);
    b.b6 = cv.take<double2>((size_t)nI * n6);
    b.coef = cv.take<double2>(3 * (size_t)Ltot);
    return b;
}

size_t chunk_bytes(const std::vector<Item*>& items, int Mx, int My) {
    int Ltot = 0, maxZS1 = 0;
    for (auto* it : items) {
        Ltot += it->Z;
        maxZS1 = std::max(maxZS1, it->Z * it->S1);
    }
    Carve cv;
    carve_chunk(cv, (int)items.size(), Ltot, maxZS1, Mx, My);
    return cv.off;
}

sc_status solve_chunk(sc_context* ctx, std::vector<Item*> items, int Mx, int My, cudaStream_t st,
                      const GemmEngine& eng, int* status, double* stage_ms) {
    Workspace& ws = ctx->ws;
    // deepest stacks first: the instances still inside their stack at depth
    // step j are then items[0 .. active(j))
    std::stable_sort(items.begin(), items.end(), [](const Item* a, const Item* b) { return a->Z > b->Z; });
    const int nI = (int)items.size();
    const int MF = Mx * My, n2 = 2 * MF, n4 = 4 * MF, n6 = 6 * MF;
    const long long s4 = (long long)n4 * n4, s6 = (long long)n6 * n6, sX = (long long)n4 * 3 * MF;
    int Ltot = 0, maxZS1 = 0;
    std::vector<int> off(nI);
    for (int a = 0; a < nI; ++a) {
        off[a] = Ltot;
        Ltot += items[a]->Z;
        maxZS1 = std::max(maxZS1, items[a]->Z * items[a]->S1);
    }
    const int maxZ = items[0]->Z;
    Carve cv;
    carve_chunk(cv, nI, Ltot, maxZS1, Mx, My);
    char* base = nullptr;
    SC_TRY(ws.get(&base, cv.off, WS_SWEEP, st));
    Carve real;
    real.base = base;
    ChunkBufs b = carve_chunk(real, nI, Ltot, maxZS1, Mx, My);
    // device pointer tables: chain (maxZ * nI * CHAIN_PTRS), final copies (2 nI), outputs (2 nI)
    constexpr int CHAIN_PTRS = 9;
    const size_t nptr = (size_t)maxZ * nI * CHAIN_PTRS + 4 * (size_t)nI;
    void** dptr = nullptr;
    SC_TRY(ws.get(&dptr, nptr, WS_SWEEP_PTR, st));

    // host-built per-instance and per-layer tables
    std::vector<double> hlat((size_t)nI * (Mx + My)), hkinv(nI), hkz0(2 * (size_t)nI), kdz(Ltot);
    std::vector<int> hinst(Ltot);
    std::vector<cplx> hsv((size_t)nI * 7 * MF);
    for (int a = 0; a < nI; ++a) {
        const VolumePlan& P = items[a]->plan;
        const double k = P.dims.k;
        for (int i = 0; i < Mx; ++i) hlat[(size_t)a * (Mx + My) + i] = P.up[i];
        for (int i = 0; i < My; ++i) hlat[(size_t)a * (Mx + My) + Mx + i] = P.wq[i];
        hkinv[a] = 1.0 / (k * k);
        hkz0[2 * a] = k;
        hkz0[2 * a + 1] = P.z[0];
        const int Z = items[a]->Z;
        // layer thickness as the reference's Gd/Gc scales use it (ScatterVolume.cpp:297-321)
        for (int l = 0; l < Z; ++l) {
            const double dz = (Z == 1) ? P.z[Z] - P.z[0] : P.z[l + 1] - P.z[l];
            kdz[off[a] + l] = k * dz;
            hinst[off[a] + l] = a;
        }
        cplx* sv = hsv.data() + (size_t)a * 7 * MF;
        std::copy(P.Sx.begin(), P.Sx.end(), sv);
        std::copy(P.Sy.begin(), P.Sy.end(), sv + MF);
        std::copy(P.Sz0.begin(), P.Sz0.end(), sv + 2 * MF);
        std::copy(P.Sz1.begin(), P.Sz1.end(), sv + 3 * MF);
        std::copy(P.EF.begin(), P.EF.end(), sv + 4 * MF);
    }
    // the reduced boundary system divides by Sz0 at every order
    bool reduced = true;
    for (int a = 0; a < nI && reduced; ++a)
        for (const cplx& z : items[a]->plan.Sz0)
            if (std::abs(z) < 1e-9) reduced = false;
    // chain step j for instance a (layer l, counted from the bottom of its stack):
    // operands of the four products and the mix in between, and t = i kdz_l.
    // U and V live in the transfer scratch, free once the layer factors exist.
    const long long n2sq = (long long)n2 * n2, suv = 2LL * n2 * 3 * MF;
    std::vector<const void*> hptr(nptr);
    std::vector<double2> htv((size_t)maxZ * nI, make_double2(0.0, 0.0));
    for (int j = 0; j < maxZ; ++j) {
        const void** row = hptr.data() + (size_t)j * nI * CHAIN_PTRS;
        int act = 0;
        while (act < nI && items[act]->Z > j) ++act;
        for (int a = 0; a < act; ++a) {
            const int l = off[a] + items[a]->Z - 1 - j;
            const double2* Tl = b.T + l * s4;                 // F | G B | C G
            double2* Xc = ((j & 1) ? b.X1 : b.X0) + a * sX;
            double2* Xn = ((j & 1) ? b.X0 : b.X1) + a * sX;
            double2* U = b.scr + a * suv;
            double2* V = U + (long long)n2 * 3 * MF;
            row[0 * nI + a] = Tl + n2sq;          // G B
            row[1 * nI + a] = Xc + n2;            // X2
            row[2 * nI + a] = U;
            row[3 * nI + a] = Tl;                 // F
            row[4 * nI + a] = Xc;                 // X1 (and the whole of X for the mix)
            row[5 * nI + a] = V;
            row[6 * nI + a] = Xn;                 // X1'
            row[7 * nI + a] = Tl + 2 * n2sq;      // C G
            row[8 * nI + a] = Xn + n2;            // X2'
            htv[(size_t)j * nI + a] = make_double2(0.0, kdz[l]);
        }
    }
    double2* dtv = nullptr;
    SC_TRY(ws.get(&dtv, htv.size(), WS_CHAIN_T, st));
    SC_CUDA_TRY(cudaMemcpyAsync(dtv, htv.data(), sizeof(double2) * htv.size(), cudaMemcpyHostToDevice, st));
    const void** tail = hptr.data() + (size_t)maxZ * nI * CHAIN_PTRS;
    for (int a = 0; a < nI; ++a) {
        tail[a] = ((items[a]->Z & 1) ? b.X1 : b.X0) + a * sX;
        tail[nI + a] = b.A6 + a * s6 + (long long)3 * MF * n6 + 2 * MF;
        tail[2 * nI + a] = b.b6 + (long long)a * n6;
        tail[3 * nI + a] = items[a]->x;
    }
    SC_CUDA_TRY(cudaMemcpyAsync(b.lat, hlat.data(), sizeof(double) * hlat.size(), cudaMemcpyHostToDevice, st));
    SC_CUDA_TRY(cudaMemcpyAsync(b.kinv, hkinv.data(), sizeof(double) * nI, cudaMemcpyHostToDevice, st));
    SC_CUDA_TRY(cudaMemcpyAsync(b.kz0, hkz0.data(), sizeof(double) * 2 * nI, cudaMemcpyHostToDevice, st));
    SC_CUDA_TRY(cudaMemcpyAsync(b.inst, hinst.data(), sizeof(int) * Ltot, cudaMemcpyHostToDevice, st));
    SC_CUDA_TRY(cudaMemcpyAsync(b.svec, hsv.data(), sizeof(cplx) * hsv.size(), cudaMemcpyHostToDevice, st));
    SC_CUDA_TRY(cudaMemcpyAsync(dptr, hptr.data(), sizeof(void*) * nptr, cudaMemcpyHostToDevice, st));
    SC_CUDA_TRY(cudaMemsetAsync(b.info, 0, sizeof(int) * nI, st));

    cudaEvent_t* ev = ctx->ev;
    SC_CUDA_TRY(cudaEventRecord(ev[0], st));
    // 1. Fourier coefficients of every slice
    for (int a = 0; a < nI; ++a) {
        const Item* it = items[a];
        SC_TRY(fft2_crop(st, it->sample, it->Z, it->S1, it->S2, Mx, My, b.Nf + (long long)off[a] * MF,
                         b.Nif + (long long)off[a] * MF, b.R2, b.Ri2, b.bins));
    }
    SC_CUDA_TRY(cudaEventRecord(ev[1], st));
    // 2. B, C, Omega
    const long long s2 = (long long)n2 * n2;
    SC_TRY(assemble_bc_layers(st, b.Nf, b.Nif, Ltot, Mx, My, b.lat, b.inst, b.kinv, b.B, b.C));
    {
        GemmArgs g;
        g.m = g.n = g.k = n2;
        g.A = b.B;
        g.lda = n2;
        g.sA = s2;
        g.B = b.C;
        g.ldb = n2;
        g.sB = s2;
        g.C = b.Om;
        g.ldc = n2;
        g.sC = s2;
        SC_TRY(eng.run(st, g, Ltot));
    }
    SC_CUDA_TRY(cudaEventRecord(ev[2], st));
    // 3. inverse layer factors
    int squarings = 0;
    SC_TRY(transfer_inv_batched(st, eng, n2, Ltot, b.B, b.C, b.Om, kdz, b.T, b.scr, b.dnorm, b.coef, &squarings));
    SC_CUDA_TRY(cudaEventRecord(ev[3], st));
    // 4. chain from f3 up through each stack
    SC_TRY(boundary_f3(st, MF, b.svec, 7LL * MF, b.X0, sX, nI));
    const unsigned chain_blocks = (unsigned)std::min<long long>(1024, ((long long)n2 * 3 * MF + 255) / 256);
    for (int j = 0; j < maxZ; ++j) {
        int act = 0;
        while (act < nI && items[act]->Z > j) ++act;
        void** row = dptr + (size_t)j * nI * CHAIN_PTRS;
        auto cpt = [&](int k) { return reinterpret_cast<const double2* const*>(row + (size_t)k * nI); };
        auto mpt = [&](int k) { return reinterpret_cast<double2* const*>(row + (size_t)k * nI); };
        auto prod = [&](int a, int lda, int bb, int ldb, int c, int ldc, double beta) {
            GemmArgs g;
            g.m = n2;
            g.n = 3 * MF;
            g.k = n2;
            g.beta = make_double2(beta, 0.0);
            g.Ap = cpt(a);
            g.lda = lda;
            g.Bp = cpt(bb);
            g.ldb = ldb;
            g.Cp = mpt(c);
            g.ldc = ldc;
            return eng.run(st, g, act);
        };
        SC_TRY(prod(0, n2, 1, n4, 2, n2, 0.0));                 // U = (G B) X2
        SC_TRY(prod(3, n2, 4, n4, 5, n2, 0.0));                 // V = F X1
        chain_mix_kernel<<<dim3(chain_blocks, act), 256, 0, st>>>(n2, 3 * MF, dtv + (size_t)j * nI, mpt(2), mpt(5),
                                                                  cpt(4), mpt(6));
        count_launch();
        SC_CHECK_LAUNCH("chain_mix");
        SC_TRY(prod(3, n2, 5, n2, 6, n4, -1.0));                // X1' = F (2 V - t U) - X1
        SC_TRY(prod(7, n2, 2, n2, 8, n4, 1.0));                 // X2' = X2 + (C G)((t^2/2) U - t V)
    }
    SC_CUDA_TRY(cudaEventRecord(ev[4], st));
    // 5. boundary systems and their solves: with R eliminated order by order
    // (3MF unknowns) when no order grazes the top interface, else the full
    // 6MF system of ScatterVolume.cpp:398-466
    void** tl = dptr + (size_t)maxZ * nI * CHAIN_PTRS;
    const auto* Yp = reinterpret_cast<const double2* const*>(tl);
    if (reduced) {
        const int n3 = 3 * MF;
        const long long s3 = (long long)n3 * n3;
        SC_TRY(boundary_reduced(st, MF, b.svec, 7LL * MF, b.kz0, Yp, n4, b.A6, s3, b.b6, n3, nI));
        SC_TRY(getrf(st, b.A6, n3, s3, n3, nI, b.piv, b.info));
        SC_TRY(getrs(st, b.A6, n3, s3, n3, b.piv, b.b6, n3, n3, 1, nI));
        SC_TRY(boundary_recover(st, MF, b.svec, 7LL * MF, b.kz0, Yp, n4, b.b6, n3,
                                reinterpret_cast<double2* const*>(tl + 3 * nI), nI));
    } else {
        SC_TRY(copy_blocks(st, n4, 3 * MF, Yp, n4, reinterpret_cast<double2* const*>(tl + nI), n6, nI));
        SC_TRY(boundary_system(st, MF, b.svec, 7LL * MF, b.kz0, b.A6, s6, b.b6, n6, nI));
        SC_TRY(getrf(st, b.A6, n6, s6, n6, nI, b.piv, b.info));
        SC_TRY(getrs(st, b.A6, n6, s6, n6, b.piv, b.b6, n6, n6, 1, nI));
        SC_TRY(copy_blocks(st, n6, 1, reinterpret_cast<const double2* const*>(tl + 2 * nI), n6,
                           reinterpret_cast<double2* const*>(tl + 3 * nI), n6, nI));
    }
    SC_CUDA_TRY(cudaEventRecord(ev[5], st));
    std::vector<int> hinfo(nI);
    SC_CUDA_TRY(cudaMemcpyAsync(hinfo.data(), b.info, sizeof(int) * nI, cudaMemcpyDeviceToHost, st));
    SC_CUDA_TRY(cudaStreamSynchronize(st));
    for (int i = 0; i < 5; ++i) {
        float ms = 0.f;
        SC_CUDA_TRY(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
        stage_ms[i] += ms;
    }
    for (int a = 0; a < nI; ++a) status[items[a]->idx] = hinfo[a] ? SC_SINGULAR : SC_OK;
    return SC_OK;
}

}  // namespace

sc_status sweep_solve(sc_context* ctx, int count, const sc_volume_params* params, const void* const* samples,
                      const int* Zs, const int* S1s, const int* S2s, void* const* x_out, int precision,
                      int* status, cudaStream_t st) {
    if (count < 0 || (count > 0 && (!params || !samples || !Zs || !S1s || !S2s || !x_out || !status))) {
        set_error("sweep_solve: null argument");
        return SC_BADINPUT;
    }
    int slices = -1;
    bool force = false, crt = false;
    if (precision == SC_SWEEP_FP64) {
        slices = 0;
    } else if (precision == SC_SWEEP_MIXED) {
        slices = 7;
    } else if (precision == SC_SWEEP_CRT) {
        slices = 7;
        crt = true;
    } else if ((precision & ~0xFF) == 0x100 && (precision & 0xFF) >= 1 && (precision & 0xFF) <= 7) {
        slices = precision & 0xFF;
        force = true;
    }
    if (slices < 0) {
        set_error("sweep_solve: unknown precision %d", precision);
        return SC_BADINPUT;
    }
    for (int i = 0; i < 8; ++i)
        if (!ctx->ev[i]) SC_CUDA_TRY(cudaEventCreate(&ctx->ev[i]));
    for (double& v : ctx->stage_ms) v = 0.0;
    std::vector<Item> items(count);
    std::map<std::pair<int, int>, std::vector<Item*>> groups;
    sc_status first = SC_OK;
    for (int i = 0; i < count; ++i) {
        Item& it = items[i];
        it.idx = i;
        it.Z = Zs[i];
        it.S1 = S1s[i];
        it.S2 = S2s[i];
        it.sample = static_cast<const double2*>(samples[i]);
        it.x = static_cast<double2*>(x_out[i]);
        sc_status s = make_plan(&params[i], it.Z, it.S1, it.S2, &it.plan);
        if (s == SC_OK && (!it.sample || !it.x)) {
            set_error("sweep_solve: instance %d has a null sample or output", i);
            s = SC_BADINPUT;
        }
        status[i] = s;
        if (s != SC_OK) {
            if (first == SC_OK) first = s;
            continue;
        }
        groups[{it.plan.dims.Mx, it.plan.dims.My}].push_back(&it);
    }
    // memory budget for one chunk
    size_t freeb = 0, totalb = 0;
    SC_CUDA_TRY(cudaMemGetInfo(&freeb, &totalb));
    const size_t held = ctx->ws.bytes[WS_SWEEP];
    // the int8 engines keep their packed operands in their own workspace
    // (the modular engine caps them at 8 GiB per product)
    size_t budget = (size_t)((slices ? 0.45 : 0.6) * (double)(freeb + held));
    const size_t cap = (size_t)48 << 30;
    if (budget > cap) budget = cap;
    GemmEngine eng;
    eng.slices = slices;
    eng.force_int8 = force;
    eng.force_crt = crt;
    eng.ws = &ctx->ws;
    SC_TRY(ctx->ws.get(&eng.err, 1, WS_OZ_ERR, st));
    SC_CUDA_TRY(cudaMemsetAsync(eng.err, 0, sizeof(int), st));
    const auto t0 = ctx->ev[7];
    SC_CUDA_TRY(cudaEventRecord(t0, st));
    double stage[8] = {};
    for (auto& kv : groups) {
        const int Mx = kv.first.first, My = kv.first.second;
        auto& list = kv.second;
        std::stable_sort(list.begin(), list.end(), [](const Item* a, const Item* b) { return a->Z > b->Z; });
        size_t pos = 0;
        while (pos < list.size()) {
            std::vector<Item*> chunk{list[pos]};
            size_t nxt = pos + 1;
            while (nxt < list.size()) {
                chunk.push_back(list[nxt]);
                if (chunk_bytes(chunk, Mx, My) > budget) {
                    chunk.pop_back();
                    break;
                }
                ++nxt;
            }
            if (chunk_bytes(chunk, Mx, My) > budget) {
                set_error("sweep_solve: instance %d (M = %dx%d, %d layers) exceeds the device memory budget",
                          chunk[0]->idx, Mx, My, chunk[0]->Z);
                status[chunk[0]->idx] = SC_OOM;
                if (first == SC_OK) first = SC_OOM;
                pos = nxt;
                continue;
            }
            SC_TRY(solve_chunk(ctx, chunk, Mx, My, st, eng, status, stage));
            pos = nxt;
        }
    }
    SC_CUDA_TRY(cudaEventRecord(ctx->ev[6], st));
    SC_CUDA_TRY(cudaEventSynchronize(ctx->ev[6]));
    float total = 0.f;
    SC_CUDA_TRY(cudaEventElapsedTime(&total, t0, ctx->ev[6]));
    for (int i = 0; i < 5; ++i) ctx->stage_ms[i] = stage[i];
    ctx->stage_ms[7] = total;
    if (slices) {
        int herr = 0;
        SC_CUDA_TRY(cudaMemcpy(&herr, eng.err, sizeof(int), cudaMemcpyDeviceToHost));
        if (herr) {
            set_error("sweep_solve: tensor-core pipeline wait timed out (stage %d)", herr);
            return SC_CUDA_ERROR;
        }
    }
    for (int i = 0; i < count && first == SC_OK; ++i)
        if (status[i] != SC_OK) {
            first = (sc_status)status[i];
            set_error("sweep_solve: instance %d failed (status %d)", i, status[i]);
        }
    return first;
}

}  // namespace sc
