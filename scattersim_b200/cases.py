"""Named solve workloads, for timing and profiling one configuration at a time.

    python -m scattersim_b200.cases <case> [repeats]

Cases (seeded synthetic samples, see samples.py):
  thin          64x64 triangle map, 10x10 um, 1 um slab, lambda 0.5, 11x11 orders
  volume        128x128x32 sphere volume, 20x20x8 um, lambda 0.6, 10 deg, 21x21 orders
  volume8       the same geometry with 8 slices
  small         128x128x4 sphere volume, 11x11 orders (a short QR capture)
  fp64          measured FP64 throughput: FMA pipe and mma.sync f64
  sweep [n]     the uneven sweep (first n of 256 instances: 64 wavelengths x 4
                angles, 4-16 layer disk stacks, 7..25 orders) in one batched call
  sweep_mixed [n]  the sweep with the mixed path (int8 tensor-core products, 7
                   digit slices, where the autotuner finds them faster)
  sweep_plain [n]  the same instances, one per-instance solve each
    (sweep cases accept --choices-out FILE to save the GEMM autotuner's table
     and --choices-in FILE to replay one, e.g. under a profiler)
  volume31      the sphere volume at 31x31 orders (M = 961, 3844 x 3844 layer
                matrices), solved in FP64 and in mixed precision; prints times
                and the mixed path's error per stage against the FP64 path
  fno_train     20 surrogate training steps (batch 64, random maps and targets):
                samples/s and the launch mix of the network's kernels
  gemm          batched complex GEMM throughput at the shapes of the solves
  gemm_int8     one int8 digit-sliced GEMM shape (1250^3 x 8) at 7 then 4 slices,
                twice each (the profiling case of the tcgen05 MMA kernel)
  layer [N]     scatterlayer's default stack (4 layers) under an N x N polar beam
                (default 1024: 1,048,576 waves) and a 15-layer stack under a
                256 x 256 beam: waves/s of the beam and of the batched layer
                solve (bench.py --workload layer adds the host baseline)
Prints the per-stage device milliseconds of the last repeat.
"""
from __future__ import annotations

import math
import sys

D10 = (math.sin(math.radians(10.0)), 0.0, math.cos(math.radians(10.0)))


def case(name):
    from . import samples
    if name == "thin":
        return samples.triangle_map(0), dict(lambda_=0.5, size=(10.0, 10.0, 1.0), coef=(11, 11), ex=(1.0, 0.0),
                                              ey=(0.0, 0.0))
    vol = dict(lambda_=0.6, size=(20.0, 20.0, 8.0), coef=(21, 21), direction=D10, ex=(1.0, 0.0), ey=(0.0, 0.0))
    if name == "volume":
        return samples.sphere_volume(0), vol
    if name == "volume8":
        return samples.sphere_volume(0, nz=8), vol
    if name == "small":
        return samples.sphere_volume(0, nz=4), dict(vol, coef=(11, 11))
    raise KeyError(name)


def main(argv):
    import torch
    from . import solver
    name = argv[1] if len(argv) > 1 else "thin"
    reps = int(argv[2]) if len(argv) > 2 else 1
    if name == "fp64":
        ctx = solver.Context(0)
        print(f"fp64 FMA pipe {ctx.fp64_peak_tflops():.2f} TFLOP/s, mma.sync f64 {ctx.fp64_peak_tflops(True):.2f} TFLOP/s")
        ctx.close()
        return 0
    if name == "gemm":
        return gemm_case()
    if name == "volume31":
        return volume31_case()
    if name == "fno_train":
        return fno_train_case()
    if name == "gemm_int8":
        return gemm_int8_case()
    if name == "layer":
        return layer_case(int(argv[2]) if len(argv) > 2 else 1024)
    if name in ("sweep", "sweep_plain", "sweep_mixed"):
        count = int(argv[2]) if len(argv) > 2 and not argv[2].startswith("--") else 256
        opt = dict(zip(argv[3::2], argv[4::2])) if len(argv) > 3 else {}
        return sweep_case(name, count, opt.get("--choices-in"), opt.get("--choices-out"))
    smp, kw = case(name)
    ctx = solver.Context(0)
    p = solver.make_params(**kw)
    d = torch.from_numpy(smp).cuda()
    for _ in range(reps):
        solver.solve(ctx, p, d)
    torch.cuda.synchronize()
    print(name, {k: round(v, 3) for k, v in ctx.stage_ms().items()}, "launches", ctx.launches())
    ctx.close()
    return 0


def gemm_case():
    import ctypes
    import torch
    from . import solver
    from ._lib import check
    ctx = solver.Context(0)
    one = (ctypes.c_double * 2)(1.0, 0.0)
    zero = (ctypes.c_double * 2)(0.0, 0.0)
    for m, n, k, batch in [(98, 98, 98, 512), (242, 242, 242, 256), (450, 450, 450, 128), (882, 882, 882, 64),
                           (1250, 1250, 1250, 32), (1764, 1764, 1764, 8), (2500, 1875, 2500, 8),
                           (3528, 3528, 3528, 2)]:
        A = torch.randn(batch, k, m, dtype=torch.complex128, device="cuda")
        B = torch.randn(batch, n, k, dtype=torch.complex128, device="cuda")
        C = torch.empty(batch, n, m, dtype=torch.complex128, device="cuda")
        args = (ctx.handle, m, n, k, one, ctypes.c_void_p(A.data_ptr()), m, m * k, ctypes.c_void_p(B.data_ptr()), k,
                k * n, zero, ctypes.c_void_p(C.data_ptr()), m, m * n, batch, None)
        for _ in range(2):
            check(ctx.lib.sc_zgemm_batched(*args))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        reps = 5
        for _ in range(reps):
            check(ctx.lib.sc_zgemm_batched(*args))
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / reps
        tf = 8.0 * m * n * k * batch / (ms * 1e-3) / 1e12
        ref = (A[0].T @ B[0].T).T   # column-major product of batch 0
        err = (C[0] - ref).abs().max().item() / ref.abs().max().item()
        print(f"zgemm m={m} n={n} k={k} batch={batch}: {ms:.3f} ms, {tf:.1f} TFLOP/s, err {err:.1e}")
        for slices in (4, 6, 7):
            eargs = (ctx.handle, slices) + args[1:]
            check(ctx.lib.sc_zgemm_emulated_batched(*eargs))
            e0.record()
            for _ in range(reps):
                check(ctx.lib.sc_zgemm_emulated_batched(*eargs))
            e1.record()
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / reps
            tf = 8.0 * m * n * k * batch / (ms * 1e-3) / 1e12
            err = (C[0] - ref).abs().max().item() / ref.abs().max().item()
            print(f"   int8 x{slices}: {ms:.3f} ms, {tf:.1f} FP64-equivalent TFLOP/s, err {err:.1e}")
    ctx.close()
    return 0


def fno_train_case(steps=20, batch=64):
    import time
    import numpy as np
    import torch
    from . import surrogate as sg
    rng = np.random.default_rng(0)
    sur = sg.Surrogate(0, max_batch=batch, seed=1)
    maps = torch.from_numpy(rng.uniform(1.0, 1.6, (batch, 64, 64)).astype(np.float32)).cuda()
    lams = torch.from_numpy(rng.uniform(0.4, 0.8, batch).astype(np.float32)).cuda()
    tgt = torch.from_numpy(rng.standard_normal((batch, sg.NOUT)).astype(np.float32)).cuda()
    sur.train_step(maps, lams, tgt, 1e-4)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        sur.train_step(maps, lams, tgt, 1e-4)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    print(f"fno_train: {steps * batch / dt:.0f} samples/s ({1e3 * dt / steps:.2f} ms per step of {batch})")
    sur.close()
    return 0


def volume31_case(N=64):
    """Mixed precision at 31x31 orders, error per stage against the FP64 path."""
    import json
    import time
    import numpy as np
    import torch
    from . import samples, solver
    from ._lib import SC_SWEEP_FP64, SC_SWEEP_MIXED
    smp = samples.sphere_volume(0)
    kw = dict(lambda_=0.6, size=(20.0, 20.0, 8.0), coef=(31, 31), direction=D10, ex=(1.0, 0.0), ey=(0.0, 0.0))
    p = solver.make_params(**kw)
    d = torch.from_numpy(smp).cuda()
    ctx = solver.Context(0)
    # x-z slice through the volume centre: 6 um of z around the slab, 20 um of x
    i = np.arange(N)
    zz, xx = np.meshgrid(-6.0 + 12.0 * i / (N - 1), 20.0 * i / (N - 1), indexing="ij")
    pts = torch.from_numpy(np.stack([xx.ravel(), np.full(N * N, 10.0), zz.ravel()], -1)).cuda()
    out = {}
    sols = {}
    for name, prec in (("fp64", SC_SWEEP_FP64), ("mixed", SC_SWEEP_MIXED)):
        ctx.set_precision(prec)
        solver.solve(ctx, p, d)              # warm-up (allocations, GEMM autotuning)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        sol = solver.solve(ctx, p, d)
        torch.cuda.synchronize()
        out[f"{name}_solve_s"] = time.perf_counter() - t0
        out[f"{name}_stage_ms"] = {k: round(v, 1) for k, v in ctx.stage_ms().items()}
        wt = solver.waves(ctx, p, sol)
        E64 = solver.evaluate(ctx, wt.E0, wt.k, wt.z_layers, wt.begin, wt.end, pts, precision=0)
        E32 = solver.evaluate(ctx, wt.E0, wt.k, wt.z_layers, wt.begin, wt.end, pts, precision=1)
        sols[name] = (sol.x.cpu().numpy(), sol.Qc.cpu().numpy(), sol.Qh.cpu().numpy(), E64.cpu().numpy(),
                      E32.cpu().numpy())
        del wt
    ctx.set_precision(SC_SWEEP_FP64)

    def rel(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    f, m = sols["fp64"], sols["mixed"]
    out["err_vs_fp64"] = {"R/T x": rel(m[0], f[0]), "interior Qc": rel(m[1], f[1]), "interior Qh": rel(m[2], f[2]),
                          "field, FP64 evaluator": rel(m[3], f[3]),
                          "field, FP32 evaluator (FP64 phase reduction)": rel(m[4], f[3]),
                          "FP32 evaluator alone on the FP64 waves": rel(f[4], f[3])}
    print(json.dumps(out))
    ctx.close()
    return 0


def gemm_int8_case():
    import ctypes
    import torch
    from . import solver
    from ._lib import check
    ctx = solver.Context(0)
    m = n = k = 1250
    batch = 8
    A = torch.randn(batch, k, m, dtype=torch.complex128, device="cuda")
    B = torch.randn(batch, n, k, dtype=torch.complex128, device="cuda")
    C = torch.empty(batch, n, m, dtype=torch.complex128, device="cuda")
    one = (ctypes.c_double * 2)(1.0, 0.0)
    zero = (ctypes.c_double * 2)(0.0, 0.0)
    for s in (7, 4):
        args = (ctx.handle, s, m, n, k, one, ctypes.c_void_p(A.data_ptr()), m, m * k, ctypes.c_void_p(B.data_ptr()),
                k, k * n, zero, ctypes.c_void_p(C.data_ptr()), m, m * n, batch, None)
        for _ in range(2):
            check(ctx.lib.sc_zgemm_emulated_batched(*args))
    torch.cuda.synchronize()
    print("gemm_int8 done")
    ctx.close()
    return 0


def sweep_case(name, count, choices_in=None, choices_out=None):
    import time
    import torch
    from . import samples, solver
    inst = samples.sweep_instances(0, count=count)
    params = [solver.make_params(**it.params_kw()) for it in inst]
    smp = [torch.from_numpy(it.maps).cuda() for it in inst]
    ctx = solver.Context(0)
    if choices_in:
        import json
        with open(choices_in) as f:
            ctx.set_gemm_choices(json.load(f))
    layers = sum(it.maps.shape[0] for it in inst)
    orders = {}
    for it in inst:
        orders[it.orders] = orders.get(it.orders, 0) + 1
    print(f"{count} instances, {layers} layers, orders {dict(sorted(orders.items()))}")
    for rep in range(2):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if name == "sweep":
            solver.sweep(ctx, params, smp)
        elif name == "sweep_mixed":
            solver.sweep(ctx, params, smp, precision=1)
        else:
            for p, s in zip(params, smp):
                solver.solve(ctx, p, s, fields=False)
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        print(f"{name} rep {rep}: {dt:.3f} s, {count / dt:.2f} solves/s")
    if name != "sweep_plain":
        print({k: round(v, 1) for k, v in ctx.stage_ms().items()})
    if choices_out:
        import json
        with open(choices_out, "w") as f:
            json.dump(ctx.gemm_choices(), f)
    ctx.close()
    return 0




def layer_case(N=1024, reps=5):
    """Batched homogeneous-layer solves: device time per call (CUDA events), waves/s."""
    import numpy as np
    import torch

    from . import layers, solver
    ctx = solver.Context(0)
    stacks = [("scatterlayer defaults (4 layers)", dict(n=(1, 1.4, 1.4, 1.0), kappa=(0.05,), z=(-3.0, 0.0, 3.0)), N),
              ("15 layers", dict(n=[1.0] + [1.2 + 0.05 * i for i in range(14)], kappa=[0.01] * 14,
                                 z=[-3.0 + 0.4 * i for i in range(14)]), 256)]
    for label, st, nb in stacks:
        L, n, kappa, z = layers.fill_layers(st["n"], st["kappa"], st["z"])
        kc, e = layers._centre(1.0, (0, 0, 1), (0, 0), (1, 0), (0, 0), n[0])
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        tb, ts = [], []
        for r in range(reps + 2):
            ev[0].record()
            ks, Es = layers.beam(ctx, 1.0, kc, e, 1.0, 0.0, (nb, nb))
            ev[1].record()
            out = layers.layer_solve(ctx, ks, Es, n, kappa, z, 1.0)
            ev[2].record()
            torch.cuda.synchronize()
            if r >= 2:
                tb.append(ev[0].elapsed_time(ev[1]))
                ts.append(ev[1].elapsed_time(ev[2]))
        W = nb * nb
        tbm, tsm = float(np.median(tb)), float(np.median(ts))
        flops = W * (8.0 / 3.0) * (6 * L) ** 3          # LU of the 6L x 6L complex system
        print(f"{label}: {W} waves; beam {tbm:.3f} ms ({W / tbm * 1e3:.3e} waves/s); "
              f"layer solve {tsm:.3f} ms ({W / tsm * 1e3:.3e} waves/s, {flops / tsm / 1e9:.2f} TFLOP/s FP64 LU)")
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
