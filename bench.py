#!/usr/bin/env python
"""Benchmark: RCWA solves/s on B200 for the scattervolume solve.

Default workload (--workload sweep): the batched sweep of 256 uneven instances
-- 64 seeded wavelengths in [0.4, 0.8] um x incidence 0/10/20/30 deg, each a
seeded 4-16 layer stack of 64x64 random-disk maps (n 1.0-1.6, 25x25 um period,
layer thickness 0.1-0.5 um), Fourier orders drawn from {7,11,15,21,25}^2 --
solved for R/T.  One step = the whole 256-instance sweep, samples resident in
HBM.  The headline value is the batched mixed-precision path (int8 tcgen05
digit-sliced products, 7 slices, where the GEMM autotuner finds them faster);
the line also carries the batched FP64 path, the plain per-instance FP64 path
(timed on a sample stratified over every incidence angle and order count) and
the R/T error of the mixed path against FP64.  Under torchrun the one sweep is
split over the ranks (LPT by cost) and the R/T vectors are all-gathered inside
every timed step (strong scaling).

--workload volume: the plain 3-D volume -- a 128x128x32-voxel sphere volume over
20x20x8 um (seeded), 32 layers, lambda 0.6 um, 10 deg, x-polarised, 21x21
orders, FP64 with interior fields; one step = one solve.

--workload layer: scatterlayer's focused-beam solve -- the reference's default
stack (n 1, 1.4 + 0.05i, 1.4, 1; boundaries -3, 0, 3 um; lambda 1 um) under a
1024 x 1024 polar beam (alpha 1 rad about z, y-polarised): 1,048,576 incident
plane waves, one 24 x 24 complex system each; one step = the batched layer
solve of the whole beam (incident waves resident in HBM), in plane waves/s.

--workload field: the field of the solved 3-D volume above on a 512x512x64 grid
(the factorised grid evaluator, complex64 out), in plane-wave evaluations/s
(the work of the direct sum), with the direct evaluator and the 64x64 triangle
map's 256x256 x-z slice beside it.

--workload surrogate: the learned surrogate of the thin-volume solve: trains the network on
--train-solves plain solves for --epochs, then times the 2000 held-out maps with
the energy-balance fallback at several gate tolerances (the headline gate is the
fastest with p90 error <= 1e-2), beside the fallback-only and per-instance paths;
--ensemble 2 trains two networks, predicts their mean and also falls back where
they disagree.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference] [--workload sweep|volume|layer|field|surrogate]

Timing is on the device (CUDA events), max over ranks.  --workload volume and
layer run one independent instance / beam per rank under torchrun (weak
scaling).  --case NAME runs one of the named profiling cases listed below.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RCWA solves/sec at stated err vs FP64: batched/mixed/surrogate vs plain GPU"
UNIT = "solves/s"
WORKLOAD = dict(lambda_=0.6, size=(20.0, 20.0, 8.0), coef=(21, 21),
                direction=(math.sin(math.radians(10.0)), 0.0, math.cos(math.radians(10.0))),
                ex=(1.0, 0.0), ey=(0.0, 0.0), n=(1.0, 1.0))
WORKLOAD_NAME = ("plain 3-D volume: 128x128x32 seeded sphere volume over 20x20x8 um, 32 layers, "
                 "lambda 0.6 um, 10 deg, x-pol, orders 21x21 (M=441, 1764x1764 per layer), fields on")
Z_LAYERS = 32
N_2M = 2 * 441
SWEEP_NAME = ("uneven sweep: 256 instances = 64 seeded wavelengths in [0.4, 0.8] um x 0/10/20/30 deg incidence; "
              "each a seeded 4-16 layer stack of 64x64 random-disk maps (n 1.0-1.6, 25x25 um period, 0.1-0.5 um "
              "layers); orders drawn from {7,11,15,21,25}^2; x-pol; R/T only")
LAYER_METRIC = "plane waves/s through a homogeneous multilayer stack (scatterlayer focused-beam solve)"
LAYER_UNIT = "waves/s"
LAYER_BEAM = 1024
LAYER_STACK = dict(n=(1.0, 1.4, 1.4, 1.0), kappa=(0.05,), z=(-3.0, 0.0, 3.0))
LAYER_NAME = ("scatterlayer default stack (n 1, 1.4+0.05i, 1.4, 1; boundaries -3, 0, 3 um; lambda 1 um) under a "
              "1024x1024 polar beam (alpha 1 rad about z, y-pol): 1,048,576 plane waves, 24x24 complex system each")
MIXED = 1          # SC_SWEEP_MIXED: int8 tcgen05 digit-sliced products, 7 slices


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except Exception:
        return {}


def _traffic_record():
    """DRAM bytes of the QR kernel from the committed ncu summary (one capture)."""
    try:
        with open(os.path.join(ROOT, "profiles", "qr_kernel_traffic.json")) as f:
            return json.load(f)
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        if self.proc is None:
            return out
        try:
            self.proc.terminate()
            self.proc.wait(timeout=5)
        except Exception:
            pass
        rows = []
        try:
            for line in open(self.path):
                parts = [q.strip() for q in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
            os.unlink(self.path)
        except Exception:
            pass
        if not rows:
            return out
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for i, nm in enumerate(names):
                if r[5 + i].lower().startswith("active"):
                    reasons.add(nm)
        loaded = [v for v in sm if v > 600] or sm
        out.update(sm_mhz=statistics.median(loaded) if loaded else None, sm_max_mhz=max(mx) if mx else None,
                   reasons=sorted(reasons), samples=len(rows))
        return out


def cpu_layer_sample(seed=0):
    """One layer of the reference CPU path at the workload size (the oracle port).

    phi assembly, zgeev of the 1764 x 1764 layer matrix, the eigen sort and one
    T-matrix step (inverse + two products): the per-layer work of
    ScatterVolume.cpp:235-336.  Returns seconds.
    """
    from oracle import scattervolume as osv
    from scattersim_b200 import samples
    smp = samples.sphere_volume(seed)
    p = osv.Params(lambda_=WORKLOAD["lambda_"], size=WORKLOAD["size"], coef=WORKLOAD["coef"],
                   direction=WORKLOAD["direction"], ex=WORKLOAD["ex"], ey=WORKLOAD["ey"])
    d, e, dirv, k, ni, slices, num_pixels, z, M, msgs = osv.setup(smp, p)
    lat = osv.upwq_cal(M, p.size, dirv, k, ni)
    t0 = time.perf_counter()
    P, _, _ = osv.phi(slices[Z_LAYERS // 2], M, lat, k)
    w, v = osv.mkl_eigensolve(P)
    sl, sv = osv.eigen_sort(w, v)
    lam = sl
    dz = z[1] - z[0]
    odd = (np.arange(sl.size) % 2) != 0
    Gd = sv * np.where(odd, np.exp(1j * k * lam * (-dz)), 1.0)[None, :]
    Gc = sv * np.where(odd, 1.0, np.exp(1j * k * lam * dz))[None, :]
    inv = osv.mkl_inverse(Gd)
    _ = (Gc @ inv) @ Gc
    return time.perf_counter() - t0


def blas_threads():
    try:
        from threadpoolctl import threadpool_info
        info = threadpool_info()
        n = [i.get("num_threads", 0) for i in info if i.get("user_api") == "blas"]
        return max(n) if n else os.cpu_count()
    except Exception:
        return os.cpu_count()


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.workload == "sweep":
        return run_sweep_reference(args)
    if args.workload == "layer":
        return run_layer_reference(args)
    if args.workload == "field":
        return run_field_reference(args)
    if args.workload == "surrogate":
        return run_surrogate_reference(args)
    for _ in range(args.warmup):
        cpu_layer_sample(0)
    ts = [cpu_layer_sample(0) for _ in range(args.steps)]
    t_solve = Z_LAYERS * statistics.mean(ts)
    value = 1.0 / t_solve
    sample = (f"1 of {Z_LAYERS} layers per step (phi, zgeev n=1764, sort, one T-matrix step), "
              f"extrapolated x{Z_LAYERS}; numpy/scipy OpenBLAS restatement of ScatterVolume.cpp")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_solve * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD_NAME, "seed": 0},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": blas_threads(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def e2e_loop(args, ctx, params, sol, host, flush, stream, barrier, dist, world):
    """Solves/s through the public API with host buffers: pinned sample in, H2D copy,
    solve, D2H of R/T, eigenvalues and interior fields, all inside the timed region."""
    import torch
    from scattersim_b200 import solver
    pin_in = torch.from_numpy(host).pin_memory()
    outs = [torch.empty(tuple(t.shape), dtype=torch.complex128).pin_memory() for t in (sol.x, sol.evl, sol.Qc, sol.Qh)]
    h2d = pin_in.numel() * 16
    d2h = sum(o.numel() for o in outs) * 16
    barrier()
    e2e_ms = []
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        d_in = torch.empty(pin_in.shape, dtype=torch.complex128, device="cuda")
        d_in.copy_(pin_in, non_blocking=True)
        s2 = solver.solve(ctx, params, d_in)
        for o, t in zip(outs, (s2.x, s2.evl, s2.Qc, s2.Qh)):
            o.copy_(t, non_blocking=True)
        e1.record(stream)
        e1.synchronize()
        e2e_ms.append(e0.elapsed_time(e1))
    barrier()
    total = sum(e2e_ms)
    if dist is not None:
        t = torch.tensor([total], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total = float(t.item())
    return world * args.steps / (total / 1e3), h2d, d2h


def run_volume_ours(args):
    import torch
    from scattersim_b200 import samples, solver

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    ctx = solver.Context(local)
    params = solver.make_params(**WORKLOAD)
    host = samples.sphere_volume(1000 + rank)
    dev = torch.from_numpy(host).cuda()
    stream = torch.cuda.current_stream()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")   # 256 MB > 126 MB L2

    for _ in range(args.warmup):
        solver.solve(ctx, params, dev)

    # ---- device-timed steps, sample resident in HBM
    sampler = ClockSampler(local)
    barrier()
    sampler.start()
    l0 = ctx.launches()
    step_ms, qr_ms, eig_ms = [], [], []
    for _ in range(args.steps):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sol = solver.solve(ctx, params, dev)
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        st = ctx.stage_ms()
        qr_ms.append(st["qr"])
        eig_ms.append(st["eig"])
    launches = ctx.launches() - l0
    barrier()
    clocks = sampler.stop()
    total_ms = sum(step_ms)
    if dist is not None:
        t = torch.tensor([total_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
    value = world * args.steps / (total_ms / 1e3)

    # ---- end to end through the public API with host buffers
    e2e_value, h2d, d2h = None, 0, 0
    if not args.no_e2e:
        e2e_value, h2d, d2h = e2e_loop(args, ctx, params, sol, host, flush, stream, barrier, dist, world)

    # ---- roofline of the dominant kernel (the QR iteration, FP64)
    fp64_peak = ctx.fp64_peak_tflops()
    qr_flops = Z_LAYERS * 80.0 * N_2M ** 3          # 80 n^3 real flops per n x n complex Schur + vectors
    qr_s = statistics.mean(qr_ms) / 1e3
    achieved = qr_flops / qr_s / 1e12
    tr = _traffic_record()
    roofline = {"bound": "tensor", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": achieved / fp64_peak if fp64_peak else None,
                "traffic": (tr or {}).get("bytes_per_launch"),
                "kernel": "hqr_kernel (complex QR to Schur form, FP64)",
                "peak_source": "FP64 FMA probe measured in this run (MEASURED_PEAKS.json has no FP64 entry)",
                "work": f"{Z_LAYERS} x 80 n^3 flops, n = 2M = {N_2M}",
                "qr_ms": statistics.mean(qr_ms), "eig_stage_ms": statistics.mean(eig_ms)}

    line = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            t_layer = cpu_layer_sample(0)
            cpu = {"value": 1.0 / (Z_LAYERS * t_layer), "unit": UNIT, "cores": blas_threads(), "kind": "port",
                   "sample": f"1 of {Z_LAYERS} layers (phi, zgeev n=1764, sort, one T-matrix step) on the "
                             f"host cores in {t_layer:.1f} s, extrapolated x{Z_LAYERS}"}
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": WORKLOAD_NAME, "seed": "1000+rank", "l2": "flushed between steps "
                           "(256 MB write, untimed)", "parallelism": f"independent instance per rank x{world}",
                           "fields": True},
                "clocks": clocks, "gpu_launches": launches, "roofline": roofline, "cpu_baseline": cpu,
                "e2e": ({"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h}
                        if e2e_value is not None else None),
                "stage_ms": {k: round(v, 3) for k, v in ctx.stage_ms().items()}}
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# --------------------------------------------------------------------------- sweep
SWEEP_SEED = 1000
ANGLES = (0.0, 10.0, 20.0, 30.0)
ORDERS = (7, 11, 15, 21, 25)
# work of the layer-independent part of a CPU solve (the boundary zgesv of order 6M,
# Gc_static^-1 and its products) in units of one layer's work (Phi, zgeev of order
# 4M, the sort and one transfer step), from their LAPACK flop counts
FIXED_LAYERS = 0.2
PLAIN_PER_STRATUM = 2


def sweep_instances(seed=SWEEP_SEED):
    from scattersim_b200 import samples
    return samples.sweep_instances(seed, count=256)


def representatives(inst):
    """One instance per order count (the shallowest stack), the incidence angle rotating."""
    out = []
    for j, m in enumerate(ORDERS):
        cand = [it for it in inst if it.orders == m and it.angle_deg == ANGLES[j % 4]]
        out.append(min(cand, key=lambda it: (it.maps.shape[0], it.index)))
    return out


def cpu_instance_seconds(it, layers=None):
    """One whole instance through the oracle (the reference's CPU path, --external):
    Phi, zgeev of every 4M x 4M layer matrix, the sort, the transfer chain and the
    boundary zgesv (ScatterVolume.cpp:654-739).  layers: solve only the first ones."""
    from oracle import scattervolume as osv
    maps = it.maps if layers is None else it.maps[:layers]
    kw = it.params_kw()
    if layers is not None:
        kw["size"] = (it.period, it.period, it.thickness * maps.shape[0])
    t0 = time.perf_counter()
    osv.solve(maps, osv.Params(**kw), keep=False)
    return time.perf_counter() - t0


def cpu_sweep_estimate(inst, per_order):
    """Seconds of the whole sweep from per-order timings {orders: (seconds, layers solved)}:
    t_i = t_rep (L_i + FIXED_LAYERS) / (L_rep + FIXED_LAYERS)."""
    total = 0.0
    for it in inst:
        t, L = per_order[it.orders]
        total += t * (it.maps.shape[0] + FIXED_LAYERS) / (L + FIXED_LAYERS)
    return total


def cpu_sweep_baseline(inst, budget_s=25.0):
    """The GPU arm's host baseline: whole representative instances while the budget lasts,
    then one-layer instances of the remaining (larger) order counts."""
    per, spent, parts = {}, 0.0, []
    for it in representatives(inst):
        L = it.maps.shape[0] if spent < budget_s / 3 else 1
        t = cpu_instance_seconds(it, None if L == it.maps.shape[0] else L)
        per[it.orders] = (t, L)
        spent += t
        parts.append(f"{it.orders}x{it.orders}: {L} layer{'s' if L > 1 else ''} {t:.2f} s")
    total = cpu_sweep_estimate(inst, per)
    desc = ("whole scattervolume --external solves through the oracle (Phi, zgeev 4M, sort, chain, boundary "
            "zgesv), one instance per order count (" + "; ".join(parts) + f"), scaled to the sweep's "
            f"{sum(i.maps.shape[0] for i in inst)} layers by (L + {FIXED_LAYERS}) per instance")
    return len(inst) / total, desc, spent


def run_sweep_reference(args):
    """The reference's CPU path on whole instances: step j solves representative j mod 5
    (one per order count, 7..25, the shallowest stack, angles rotating) end to end."""
    inst = sweep_instances()
    reps = representatives(inst)
    warm = reps[0]
    for _ in range(args.warmup):
        cpu_instance_seconds(warm)
    times = {m: [] for m in ORDERS}
    step_s = []
    for j in range(args.steps):
        it = reps[j % len(reps)]
        t = cpu_instance_seconds(it)
        times[it.orders].append(t)
        step_s.append(t)
    per = {}
    timed = [m for m in ORDERS if times[m]]
    for m in ORDERS:
        it = reps[ORDERS.index(m)]
        if times[m]:
            per[m] = (statistics.mean(times[m]), it.maps.shape[0])
        else:   # not reached with so few steps: scale the largest timed order by (4M)^3
            mt = max(timed)
            per[m] = (statistics.mean(times[mt]) * (m / mt) ** 6, reps[ORDERS.index(mt)].maps.shape[0])
    value = len(inst) / cpu_sweep_estimate(inst, per)
    sample = ("step j = one whole instance end to end through the oracle (numpy/scipy OpenBLAS restatement of "
              "ScatterVolume.cpp: Phi, zgeev of every 4M x 4M layer matrix, sort, transfer chain, boundary zgesv, "
              "--external), cycling over one instance per order count (" +
              ", ".join(f"#{it.index}: {it.orders}x{it.orders} orders, {it.maps.shape[0]} layers, "
                        f"{it.angle_deg:g} deg" for it in reps) +
              f"); value = 256 / sum over the sweep of t(orders) (L + {FIXED_LAYERS}) / (L_rep + {FIXED_LAYERS})")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(step_s),
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": SWEEP_NAME, "seed": SWEEP_SEED},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": blas_threads(), "kind": "port", "sample": sample,
                             "per_order_s": {str(m): round(per[m][0], 3) for m in ORDERS},
                             "sample_solves_per_s": len(step_s) / sum(step_s)},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def plain_strata(inst):
    """PLAIN_PER_STRATUM instances of every (angle, orders) stratum, by index."""
    out = {}
    for it in inst:
        key = (it.angle_deg, it.orders)
        out.setdefault(key, [])
        if len(out[key]) < PLAIN_PER_STRATUM:
            out[key].append(it.index)
    return out


def run_sweep_ours(args):
    import torch
    from scattersim_b200 import solver, sweep

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev_t = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900), device_id=dev_t)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v):
        return sweep.max_over_ranks(v, dist, dev_t)

    ctx = solver.Context(local)
    inst = sweep_instances()                       # one sweep, split across the ranks
    n = len(inst)
    params = [solver.make_params(**it.params_kw()) for it in inst]
    dims = [solver.plan(p, it.maps.shape) for p, it in zip(params, inst)]
    sizes = [6 * d.MF for d in dims]
    costs = [sweep.solve_cost(it.maps.shape[0], d.MF) for it, d in zip(inst, dims)]
    parts = sweep.assign_lpt(costs, world)
    mine = parts[rank]
    dev = {i: torch.from_numpy(inst[i].maps).to(dev_t) for i in mine}
    stream = torch.cuda.current_stream()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev_t)   # 256 MB > 126 MB L2

    def solve_share(precision, samples=None):
        def fn(idx):
            smp = [samples[i] if samples is not None else dev[i] for i in idx]
            return solver.sweep(ctx, [params[i] for i in idx], smp, precision=precision).x
        return sweep.shard_solve(costs, sizes, fn, dist, dev_t)

    def timed(fn):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        return out, e0.elapsed_time(e1)

    for _ in range(args.warmup):          # the first call also autotunes every GEMM shape
        solve_share(MIXED)

    # ---- headline: batched mixed precision, device-timed, samples resident in HBM
    sampler = ClockSampler(local)
    barrier()
    sampler.start()
    l0 = ctx.launches()
    step_ms = []
    res_mixed = None
    for _ in range(args.steps):
        res_mixed, ms = timed(lambda: solve_share(MIXED))
        step_ms.append(ms)
    launches = ctx.launches() - l0
    stages = ctx.stage_ms()
    barrier()
    clocks = sampler.stop()
    total_ms = max_over_ranks(sum(step_ms))
    value = n * args.steps / (total_ms / 1e3)

    # ---- one instrumented step: per-launch GEMM timing for the roofline (not in the headline)
    ctx.kernel_timing(True)
    _, instr_ms = timed(lambda: solve_share(MIXED))
    kst = ctx.kernel_stats_ex()
    ctx.kernel_timing(False)

    # ---- batched FP64, same step count (one warm-up for its own GEMM shapes)
    solve_share(0)
    barrier()
    fp_ms = []
    res_fp = None
    for _ in range(args.steps):
        res_fp, ms = timed(lambda: solve_share(0))
        fp_ms.append(ms)
    fp_value = n * args.steps / (max_over_ranks(sum(fp_ms)) / 1e3)
    errs = [_rel(a.cpu().numpy(), b.cpu().numpy()) for a, b in zip(res_mixed, res_fp)]

    # ---- plain per-instance FP64 path on a stratified sample (every angle x order count)
    strata = plain_strata(inst)
    my_strata = [key for j, key in enumerate(sorted(strata)) if j % world == rank]
    warmed = set()
    for key in my_strata:                  # one untimed solve per order count (workspace growth)
        i = strata[key][0]
        if inst[i].orders not in warmed:
            solver.solve(ctx, params[i], torch.from_numpy(inst[i].maps).to(dev_t), fields=False)
            warmed.add(inst[i].orders)
    plain_est_ms = 0.0
    plain_count = 0
    for key in my_strata:
        ms_k = []
        for i in strata[key]:
            d_i = torch.from_numpy(inst[i].maps).to(dev_t)
            _, ms = timed(lambda: solver.solve(ctx, params[i], d_i, fields=False))
            ms_k.append(ms)
            plain_count += 1
        pop = sum(1 for it in inst if (it.angle_deg, it.orders) == key)
        plain_est_ms += pop * statistics.mean(ms_k)
    if dist is not None:       # the strata are split over the ranks: sum their estimates
        t = torch.tensor([plain_est_ms], dtype=torch.float64, device=dev_t)
        dist.all_reduce(t)
        plain_est_ms = float(t.item())
    plain_value = world * n / (plain_est_ms / 1e3)

    # ---- end to end through the public API with host buffers (same step count)
    e2e = None
    if not args.no_e2e:
        sz = [inst[i].maps.size for i in mine]
        offs = np.concatenate([[0], np.cumsum(sz)]).astype(np.int64)
        pin_in = torch.empty(int(offs[-1]), dtype=torch.complex128).pin_memory()
        for i, o in zip(mine, offs[:-1]):
            pin_in[int(o):int(o) + inst[i].maps.size].copy_(torch.from_numpy(inst[i].maps.ravel()))
        outs = [torch.empty(s, dtype=torch.complex128).pin_memory() for s in sizes]
        d_in = torch.empty_like(pin_in, device=dev_t)
        barrier()
        e2e_ms = []
        for _ in range(args.steps):
            def step():
                d_in.copy_(pin_in, non_blocking=True)
                views = {i: d_in[int(o):int(o) + inst[i].maps.size].view(inst[i].maps.shape)
                         for i, o in zip(mine, offs[:-1])}
                r = solve_share(MIXED, views)
                for o, x in zip(outs, r):
                    o.copy_(x, non_blocking=True)
                return r
            _, ms = timed(step)
            e2e_ms.append(ms)
        e2e_value = n * args.steps / (max_over_ranks(sum(e2e_ms)) / 1e3)
        e2e = {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": int(offs[-1]) * 16,
               "d2h_bytes_per_step": int(sum(sizes)) * 16}

    # ---- roofline of the dominant kernel (by device time over the instrumented step)
    peaks = _peaks()
    fp64_peak = ctx.fp64_peak_tflops()
    int8_peak_meas = ctx.int8_peak_tops() if hasattr(ctx, "int8_peak_tops") else None
    d8, dd, dc, dcg = kst["int8"], kst["dmma"], kst["crt"], kst["crt_gemm"]
    # the larger of the int8 probe and twice the measured BF16 burst peak (int8 dense is twice BF16
    # dense on B200), so that a weak probe cannot flatter the fraction
    bf16x2 = 2.0 * float(peaks.get("bf16_tflops", 1590.0))
    if int8_peak_meas and int8_peak_meas >= bf16x2:
        int8_peak, src = int8_peak_meas, ("int8 tcgen05 MMA probe measured in this run (128 x 256 x 32, "
                                          "operands resident in shared memory, no loads)")
    else:
        int8_peak, src = bf16x2, "2 x measured bf16 dense burst peak (MEASURED_PEAKS.json)"
    dom = max((("int8", d8), ("crt", dc), ("dmma", dd)), key=lambda kv: kv[1]["ms"])[0]
    if dom in ("int8", "crt"):
        st_ = d8 if dom == "int8" else dc
        achieved = st_["int8_ops"] / (st_["ms"] / 1e3) / 1e12
        tr, tr_src = None, None
        rec_name = "int8_gemm_traffic.json" if dom == "int8" else "crt_gemm_traffic.json"
        try:
            with open(os.path.join(ROOT, "profiles", rec_name)) as f:
                rec = json.load(f)
            tr = rec["bytes_per_fp64_flop"] * st_["flops"] / max(st_["launches"], 1)
            tr_src = (f"ncu dram bytes of one capture ({rec['case']}), scaled by FP64-equivalent flops per "
                      f"launch (profiles/{rec_name})")
        except Exception:
            pass
        name = ("oz_mma_kernel (int8 tcgen05 MMA, 7 digit slices, TMEM accumulators)" if dom == "int8" else
                "crt_mma_kernel (int8 tcgen05 MMA, 14 moduli, persistent 128x256 tiles, TMEM accumulators)")
        roofline = {"bound": "tensor", "achieved": achieved, "peak": int8_peak, "unit": "TOPS (int8)",
                    "frac": achieved / int8_peak, "traffic": tr, "kernel": name, "peak_source": src,
                    "launches": int(st_["launches"]), "avg_launch_ms": st_["ms"] / max(st_["launches"], 1),
                    "fp64_equivalent_tflops": st_["flops"] / (st_["ms"] / 1e3) / 1e12,
                    "fp64_peak_tflops": fp64_peak, "traffic_source": tr_src}
    else:
        achieved = dd["flops"] / (dd["ms"] / 1e3) / 1e12
        roofline = {"bound": "tensor", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                    "frac": achieved / fp64_peak, "traffic": None,
                    "kernel": "zgemm_kernel (FP64 mma.sync m8n8k4 complex GEMM)",
                    "peak_source": "FP64 FMA probe measured in this run",
                    "launches": int(dd["launches"]), "avg_launch_ms": dd["ms"] / max(dd["launches"], 1)}
    # the modular engine's whole products (exponents, packing, MMA kernel) enclose its MMA marks
    roofline["crt_whole_product_ms_per_step"] = dcg["ms"]
    roofline["crt_mma_ms_per_step"] = dc["ms"]
    if dcg["ms"] > 0:
        roofline["crt_whole_product_fp64_equivalent_tflops"] = dcg["flops"] / (dcg["ms"] / 1e3) / 1e12
    roofline["instrumented_step_ms"] = instr_ms
    roofline["gemm_time_share"] = (d8["ms"] + dd["ms"] + dcg["ms"]) / (instr_ms or 1.0)
    roofline["int8_ms_per_step"] = d8["ms"]
    roofline["fp64_tile_ms_per_step"] = dd["ms"]

    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            v, desc, spent = cpu_sweep_baseline(inst)
            cpu = {"value": v, "unit": UNIT, "cores": blas_threads(), "kind": "port",
                   "sample": desc + f"; {spent:.1f} s of host work"}
        strata_desc = (f"stratified: {PLAIN_PER_STRATUM} instances of each of the {len(strata)} (angle, orders) "
                       f"strata ({plain_count * world if world > 1 else plain_count} timed), one "
                       "sc_volume_solve (--external) each; sweep time = sum over strata of population x mean time")
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "int8 tensor products (modular, 14 moduli, or 7 digit slices, per shape) + f64",
                "data": "synthetic",
                "config": {"workload": SWEEP_NAME, "seed": SWEEP_SEED, "path": "batched mixed precision",
                           "l2": "flushed between steps (256 MB write, untimed); working set >> L2",
                           "parallelism": (f"one sweep split over {world} ranks (LPT by batched-path cost), R/T "
                                           "all-gathered inside each step" if world > 1 else "one GPU")},
                "paths": {"batched_mixed": value, "batched_fp64": fp_value,
                          "plain_fp64_per_instance": plain_value, "plain_sample": strata_desc,
                          "mixed_rt_rel_err_vs_fp64": {"max": max(errs), "median": statistics.median(errs)},
                          "speedup_mixed_vs_plain": value / plain_value,
                          "speedup_fp64_batched_vs_plain": fp_value / plain_value},
                "clocks": clocks, "gpu_launches": launches, "roofline": roofline, "cpu_baseline": cpu,
                "e2e": e2e,
                "stage_ms": {"fft": round(stages["fft"], 1), "assemble": round(stages["assemble"], 1),
                             "layer_factors": round(stages["eig"], 1), "chain": round(stages["chain"], 1),
                             "boundary": round(stages["boundary"], 1), "total": round(stages["total"], 1)}}
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def cpu_layer_waves(k, E, count):
    """The oracle's per-wave solve (ScatterLayer.cpp:110-266 restated, scipy LAPACK) on `count` waves."""
    from oracle import scatterlayer as osl
    L, n, kappa, z, ri = osl.fill_layers(LAYER_STACK["n"], LAYER_STACK["kappa"], LAYER_STACK["z"])
    t0 = time.perf_counter()
    for w in range(count):
        osl.solve_wave(k[w], E[w], ri, z, 2 * math.pi, n[0])
    return count / (time.perf_counter() - t0)


def run_layer_reference(args):
    from oracle import scatterlayer as osl
    kc, e = osl.incident(1.0, (0, 0, 1), (0, 0), (1, 0), (0, 0), LAYER_STACK["n"][0])
    ks, Es = osl.beam_polar(1.0, kc, e, 64, 64)            # a 4096-wave sample of the same beam law
    per = 2000
    for _ in range(args.warmup):
        cpu_layer_waves(ks, Es, 200)
    vals = [cpu_layer_waves(ks, Es, per) for _ in range(args.steps)]
    value = statistics.median(vals)
    sample = (f"{per} waves per step of a 64x64 beam with the workload's beam law and stack; one 24x24 complex "
              "solve per wave (numpy/scipy restatement of ScatterLayer.cpp, 1 thread like the reference's loop)")
    line = {"impl": "reference", "metric": LAYER_METRIC, "value": value, "unit": LAYER_UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per / value * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": LAYER_NAME},
            "cpu_baseline": {"value": value, "unit": LAYER_UNIT, "cores": 1, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": LAYER_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_layer_ours(args):
    import torch
    from scattersim_b200 import layers, solver

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v):
        if dist is None:
            return v
        t = torch.tensor([v], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    ctx = solver.Context(local)
    L, n, kappa, z = layers.fill_layers(LAYER_STACK["n"], LAYER_STACK["kappa"], LAYER_STACK["z"])
    kc, e = layers._centre(1.0, (0, 0, 1), (0, 0), (1, 0), (0, 0), n[0])
    ks, Es = layers.beam(ctx, 1.0, kc, e, 1.0, 0.0, (LAYER_BEAM, LAYER_BEAM))
    W = int(ks.shape[0])
    stream = torch.cuda.current_stream()
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    def timed(fn):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        return out, e0.elapsed_time(e1)

    for _ in range(args.warmup):
        layers.layer_solve(ctx, ks, Es, n, kappa, z, 1.0)
    sampler = ClockSampler(local)
    barrier()
    sampler.start()
    l0 = ctx.launches()
    step_ms = []
    for _ in range(args.steps):
        out, ms = timed(lambda: layers.layer_solve(ctx, ks, Es, n, kappa, z, 1.0))
        step_ms.append(ms)
    launches = ctx.launches() - l0
    barrier()
    clocks = sampler.stop()
    total_ms = max_over_ranks(sum(step_ms))
    value = world * W * args.steps / (total_ms / 1e3)

    # end to end: incident waves from pinned host memory, every output back to pinned host memory
    e2e = None
    if not args.no_e2e:
        hk = ks.cpu().pin_memory()
        hE = Es.cpu().pin_memory()
        dk, dE = torch.empty_like(ks), torch.empty_like(Es)
        houts = [torch.empty(o.shape, dtype=o.dtype).pin_memory() for o in out]
        barrier()
        e2e_ms = []
        for _ in range(max(1, min(3, args.steps))):
            def step():
                dk.copy_(hk, non_blocking=True)
                dE.copy_(hE, non_blocking=True)
                r = layers.layer_solve(ctx, dk, dE, n, kappa, z, 1.0)
                for h, o in zip(houts, r):
                    h.copy_(o, non_blocking=True)
                return r
            _, ms = timed(step)
            e2e_ms.append(ms)
        e2e = {"value": world * W * len(e2e_ms) / (max_over_ranks(sum(e2e_ms)) / 1e3), "unit": LAYER_UNIT,
               "h2d_bytes_per_step": int(hk.numel() * 8 + hE.numel() * 16),
               "d2h_bytes_per_step": int(sum(h.numel() for h in houts) * 16)}

    # roofline: FP64 LU of one 6L x 6L complex system per wave against the measured FP64 FMA rate
    fp64_peak = ctx.fp64_peak_tflops()
    per_ms = statistics.median(step_ms)
    flops = W * (8.0 / 3.0) * (6 * L) ** 3
    achieved = flops / (per_ms / 1e3) / 1e12
    algo_bytes = W * (24 + 48 + 4 * 3 * (L - 1) * 16)
    tr = None
    try:
        with open(os.path.join(ROOT, "profiles", "layer_solve_traffic.json")) as f:
            tr = json.load(f)["bytes_per_wave"] * W
    except Exception:
        pass
    roofline = {"bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": achieved / fp64_peak, "traffic": tr,
                "kernel": "layer_solve_kernel (one warp per wave, LU with partial pivoting in shared memory)",
                "peak_source": "FP64 FMA pipe probe measured in this run",
                "flops_per_wave": (8.0 / 3.0) * (6 * L) ** 3, "algorithmic_bytes_per_wave": algo_bytes / W,
                "hbm_gbs_achieved": algo_bytes / (per_ms / 1e3) / 1e9,
                "hbm_peak_gbs": float(_peaks().get("hbm_gbs", 6650.0))}
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            hk_np, hE_np = ks[:2000].cpu().numpy(), Es[:2000].cpu().numpy()
            v = cpu_layer_waves(hk_np, hE_np, 2000)
            cpu = {"value": v, "unit": LAYER_UNIT, "cores": 1, "kind": "port",
                   "sample": "the first 2000 waves of the workload's beam through the oracle's per-wave solve "
                             "(numpy/scipy restatement of ScatterLayer.cpp, 1 thread like the reference's loop)"}
        line = {"metric": LAYER_METRIC, "value": value, "unit": LAYER_UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": LAYER_NAME, "l2": "flushed between steps (256 MB write, untimed); "
                           "outputs 604 MB > L2", "parallelism": f"independent beam per rank x{world}"},
                "clocks": clocks, "gpu_launches": launches, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e}
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# --------------------------------------------------------------------------- field
FIELD_METRIC = "plane-wave evaluations/s of the coupled-wave field on a grid (gpuEvaluator sum)"
FIELD_UNIT = "wave-evals/s"
FIELD_NAME = ("field of the 128x128x32 sphere volume (seed 1000, 21x21 orders, 32 layers, fields on) on a "
              "512x512x64 grid (x, y in [0, 20] um, z in [-6, 6] um), complex64 out; with the 64x64 triangle "
              "map's 256x256 x-z slice (x in [0, 10], z in [-5, 5], y = 5) beside it")
FIELD_GRID = dict(origin=(0.0, 0.0, -6.0), step=(20.0 / 511, 20.0 / 511, 12.0 / 63), counts=(512, 512, 64))
THIN_GRID = dict(origin=(0.0, 5.0, -5.0), step=(10.0 / 255, 1.0, 10.0 / 255), counts=(256, 1, 256))
THIN_KW = dict(lambda_=0.5, size=(10.0, 10.0, 1.0), coef=(11, 11), ex=(1.0, 0.0), ey=(0.0, 0.0))


def wave_evals(wt, grid):
    """Sum over the grid points of the number of waves in the point's region (the direct sum's work)."""
    zl, b, e = wt.z_layers, wt.begin, wt.end
    nx, ny, nz = grid["counts"]
    total = 0
    for i in range(nz):
        z = grid["origin"][2] + grid["step"][2] * i
        l = int(sum(1 for zz in zl if z >= zz - 0.001))
        total += (int(e[l]) - int(b[l])) * nx * ny
    return total


def grid_points(grid, planes=None):
    nx, ny, nz = grid["counts"]
    o, s = grid["origin"], grid["step"]
    zs = [o[2] + s[2] * i for i in (planes if planes is not None else range(nz))]
    zz, yy, xx = np.meshgrid(np.array(zs), o[1] + s[1] * np.arange(ny), o[0] + s[0] * np.arange(nx), indexing="ij")
    return np.stack([xx.ravel(), yy.ravel(), zz.ravel()], -1)


def run_field_reference(args):
    """The evaluator sum on the host (the oracle's float64 restatement of gpuEvaluator.cu:28-68), one x-z row
    of the triangle slice's interior per step."""
    from oracle import cw as ocw
    from oracle import scattervolume as osv
    from scattersim_b200 import samples
    smp = samples.triangle_map(0)
    p = osv.Params(**THIN_KW)
    sol = osv.solve(smp, p)
    W = osv.build_waves(sol, p)
    layers = [(W.z[l], W.Pr_E[l], W.Pr_k[l], W.Pt_E[l], W.Pt_k[l]) for l in range(len(W.z))]
    zl, b, e, WE, Wk = ocw.unpack(W.Pi_E, W.Pi_k, layers)
    pts = grid_points(THIN_GRID)
    inside = pts[(pts[:, 2] > -0.5) & (pts[:, 2] < 0.5)][:64]          # points in the slab's region
    reg = ocw.region_of(inside[:, 2], zl)
    evals = int(sum(int(e[r]) - int(b[r]) for r in reg))
    for _ in range(args.warmup):
        ocw.evaluate(inside[:8], zl, b, e, WE, Wk)
    ts = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        ocw.evaluate(inside, zl, b, e, WE, Wk)
        ts.append(time.perf_counter() - t0)
    value = evals / statistics.mean(ts)
    sample = (f"{len(inside)} interior points of the 256x256 triangle-map slice ({evals} wave evaluations) per "
              "step through the oracle's float64 restatement of the evaluator sum (numpy, vectorised)")
    line = {"impl": "reference", "metric": FIELD_METRIC, "value": value, "unit": FIELD_UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(ts),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": FIELD_NAME},
            "cpu_baseline": {"value": value, "unit": FIELD_UNIT, "cores": blas_threads(), "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": FIELD_UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_field_ours(args):
    import torch
    from scattersim_b200 import samples, solver

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(v):
        if dist is None:
            return v
        t = torch.tensor([v], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    ctx = solver.Context(local)
    stream = torch.cuda.current_stream()
    params = solver.make_params(**WORKLOAD)
    vol = torch.from_numpy(samples.sphere_volume(1000 + rank)).cuda()
    sol = solver.solve(ctx, params, vol)
    wt = solver.waves(ctx, params, sol)
    evals = wave_evals(wt, FIELD_GRID)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")

    def timed(fn):
        flush.zero_()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        return out, e0.elapsed_time(e1)

    def grid_step(s=sol):
        return solver.field_grid(ctx, params, s, precision=1, **FIELD_GRID)

    for _ in range(args.warmup):
        grid_step()
    sampler = ClockSampler(local)
    barrier()
    sampler.start()
    l0 = ctx.launches()
    step_ms, stages = [], []
    for _ in range(args.steps):
        out, ms = timed(grid_step)
        step_ms.append(ms)
        stages.append(ctx.stage_ms())
    launches = ctx.launches() - l0
    barrier()
    clocks = sampler.stop()
    total_ms = max_over_ranks(sum(step_ms))
    value = world * evals * args.steps / (total_ms / 1e3)
    out_bytes = out.numel() * 8
    npts = int(np.prod(FIELD_GRID["counts"]))

    # error of the complex64 grid against the FP64 direct sum on two interior planes, and the direct
    # evaluator's own rate there (float32 with float64 phase reduction, and float64)
    planes = [22, 41]
    pts = torch.from_numpy(grid_points(FIELD_GRID, planes)).cuda()
    direct64, t64 = timed(lambda: solver.evaluate(ctx, wt.E0, wt.k, wt.z_layers, wt.begin, wt.end, pts, precision=0))
    direct32, t32 = timed(lambda: solver.evaluate(ctx, wt.E0, wt.k, wt.z_layers, wt.begin, wt.end, pts, precision=1))
    g = out[planes].reshape(-1, 3).to(torch.complex128)
    d64 = direct64.reshape(-1, 3)
    err_grid = float((g - d64).norm() / d64.norm())
    err_direct32 = float((direct32.reshape(-1, 3) - d64).norm() / d64.norm())
    g64 = solver.field_grid(ctx, params, sol, precision=0, **FIELD_GRID)[planes].reshape(-1, 3)
    err_grid64 = float((g64 - d64).norm() / d64.norm())
    plane_evals = sum((int(wt.end[l]) - int(wt.begin[l])) for l in
                      [int(sum(1 for zz in wt.z_layers if FIELD_GRID["origin"][2] + FIELD_GRID["step"][2] * i >=
                               zz - 0.001)) for i in planes]) * FIELD_GRID["counts"][0] * FIELD_GRID["counts"][1]
    direct_rate = {"float32_fp64_phase": plane_evals / (t32 / 1e3), "float64": plane_evals / (t64 / 1e3)}
    # interior planes per layer (the order-sum kernel reads each layer's mode fields once per group of up
    # to 4 of its planes)
    zls = [float(z) for z in wt.z_layers]
    per_layer = {}
    for i in range(FIELD_GRID["counts"][2]):
        zi = FIELD_GRID["origin"][2] + FIELD_GRID["step"][2] * i
        r = sum(1 for zz in zls if zi >= zz - 0.001)
        if 1 <= r <= len(zls) - 1:
            per_layer[r - 1] = per_layer.get(r - 1, 0) + 1
    plane_groups = sum((c + 3) // 4 for c in per_layer.values())
    interior_planes = sum(per_layer.values())
    del wt

    # the thin-volume slice (64x64 triangle map, 11x11 orders): factorised and direct
    tsmp = torch.from_numpy(samples.triangle_map(0)).cuda()
    tp = solver.make_params(**THIN_KW)
    tsol = solver.solve(ctx, tp, tsmp)
    twt = solver.waves(ctx, tp, tsol)
    tev = wave_evals(twt, THIN_GRID)
    solver.field_grid(ctx, tp, tsol, precision=1, **THIN_GRID)
    _, t_thin = timed(lambda: solver.field_grid(ctx, tp, tsol, precision=1, **THIN_GRID))
    tpts = torch.from_numpy(grid_points(THIN_GRID)).cuda()
    solver.evaluate(ctx, twt.E0, twt.k, twt.z_layers, twt.begin, twt.end, tpts, precision=1)
    _, t_thin_direct = timed(lambda: solver.evaluate(ctx, twt.E0, twt.k, twt.z_layers, twt.begin, twt.end, tpts,
                                                     precision=1))

    # end to end: the solution (x, eigenvalues, interior fields) from pinned host memory, the grid back
    e2e = None
    if not args.no_e2e:
        hsol = [t.cpu().pin_memory() for t in (sol.x, sol.evl, sol.Qc, sol.Qh)]
        dsol = [torch.empty_like(t) for t in (sol.x, sol.evl, sol.Qc, sol.Qh)]
        hout = torch.empty(out.shape, dtype=out.dtype).pin_memory()
        s2 = solver.VolumeSolution(sol.dims, sol.shape, *dsol)
        barrier()
        e2e_ms = []
        for _ in range(args.steps):
            def step():
                for d, h in zip(dsol, hsol):
                    d.copy_(h, non_blocking=True)
                r = grid_step(s2)
                hout.copy_(r, non_blocking=True)
                return r
            _, ms = timed(step)
            e2e_ms.append(ms)
        e2e = {"value": world * evals * args.steps / (max_over_ranks(sum(e2e_ms)) / 1e3), "unit": FIELD_UNIT,
               "h2d_bytes_per_step": int(sum(h.numel() for h in hsol) * 16),
               "d2h_bytes_per_step": int(hout.numel() * 8)}

    # roofline: the dominant stage by device time
    st = {k: statistics.mean(s[k] for s in stages) for k in ("fft", "assemble", "eig", "chain", "total")}
    names = {"fft": "boundary wave table + phase tables",
             "assemble": "order sums (field_hq_kernel from the layers' mode fields, field_h_kernel outside)",
             "eig": "y transform (field_u_kernel)", "chain": "x transform + output (field_e_kernel)"}
    MF, Mx, Ny = sol.dims.MF, sol.dims.Mx, FIELD_GRID["counts"][1]
    dom = max(("fft", "assemble", "eig", "chain"), key=lambda k: st[k])
    nz = FIELD_GRID["counts"][2]
    peak = float(_peaks().get("hbm_gbs", 6650.0))
    zb = sol.shape[0]
    # algorithmic bytes per stage: boundary wave table (3 MF waves) + the x / y phase tables; the interior
    # planes' mode fields (Qc and Qh of the layer, once per group of planes) + the slice partial sums; U
    # written; output written + U read
    bytes_dom = {"fft": 3 * MF * 96 + (FIELD_GRID["counts"][0] * Mx + FIELD_GRID["counts"][1] * sol.dims.My) * 16,
                 "assemble": plane_groups * 2 * (3 * MF * 2 * MF) * 16 + 8 * interior_planes * 3 * MF * 16,
                 "eig": nz * 3 * Mx * Ny * 16,
                 "chain": out_bytes + nz * 3 * Mx * Ny * 16}[dom]
    roofline = {"bound": "hbm", "achieved": bytes_dom / (st[dom] / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                "frac": bytes_dom / (st[dom] / 1e3) / 1e9 / peak, "traffic": None, "kernel": names[dom],
                "algorithmic_bytes": bytes_dom, "stage_ms": {names[k]: round(st[k], 3) for k in names},
                "peak_source": "MEASURED_PEAKS.json hbm_gbs" if _peaks() else "fallback 6650 GB/s"}
    if dom == "chain":
        # the x transform is FP64-bound: 3 Mx complex multiply-adds (8 flops each) per point, against the FP64
        # FMA rate measured in this run; its output write is reported beside it
        flops = 8.0 * 3 * Mx * npts
        fp64_peak = ctx.fp64_peak_tflops()
        ach = flops / (st[dom] / 1e3) / 1e12
        roofline.update({"bound": "fp64", "achieved": ach, "peak": fp64_peak, "unit": "TFLOP/s",
                         "frac": ach / fp64_peak, "algorithmic_flops": flops,
                         "peak_source": "FP64 FMA probe measured in this run",
                         "hbm_gbs_of_output_write": bytes_dom / (st[dom] / 1e3) / 1e9})
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            from oracle import cw as ocw
            E0h, Kh = twt.E0.cpu().numpy(), twt.k.cpu().numpy()
            sub = grid_points(THIN_GRID)
            sub = sub[(sub[:, 2] > -0.5) & (sub[:, 2] < 0.5)][:64]
            reg = ocw.region_of(sub[:, 2], twt.z_layers)
            ev = int(sum(int(twt.end[r]) - int(twt.begin[r]) for r in reg))
            t0 = time.perf_counter()
            ocw.evaluate(sub, twt.z_layers, twt.begin, twt.end, E0h, Kh)
            cpu = {"value": ev / (time.perf_counter() - t0), "unit": FIELD_UNIT, "cores": blas_threads(),
                   "kind": "port", "sample": f"{len(sub)} interior points of the triangle slice, {ev} wave "
                                             "evaluations, oracle float64 sum (numpy)"}
        line = {"metric": FIELD_METRIC, "value": value, "unit": FIELD_UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64 (complex64 output)", "data": "synthetic",
                "config": {"workload": FIELD_NAME, "points": npts, "wave_evals_per_step": evals,
                           "l2": "flushed between steps (256 MB write, untimed); output 403 MB > L2",
                           "parallelism": f"independent volume per rank x{world}"},
                "paths": {"grid_factorised_ms": total_ms / args.steps,
                          "grid_error_vs_fp64_direct": {"complex64_out": err_grid, "complex128_out": err_grid64},
                          "direct_evaluator_wave_evals_per_s": direct_rate,
                          "direct_float32_error_vs_fp64": err_direct32,
                          "thin_slice": {"points": 65536, "wave_evals": tev, "factorised_ms": t_thin,
                                         "direct_float32_ms": t_thin_direct,
                                         "factorised_wave_evals_per_s": tev / (t_thin / 1e3),
                                         "direct_wave_evals_per_s": tev / (t_thin_direct / 1e3)}},
                "clocks": clocks, "gpu_launches": launches, "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e}
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


# --------------------------------------------------------------------------- surrogate
SUR_METRIC = "RCWA solves/sec at stated err vs FP64: surrogate with energy-balance fallback (FNO surrogate of the thin-volume solve)"
SUR_NAME = ("FNO surrogate (4 spectral layers, width 64, 16x16 modes) of the thin-volume solve: 64x64 seeded "
            "disk/triangle maps (n 1.0-1.6, 10x10 um, 1 um slab), lambda 0.4-0.8 um, 11x11 orders; trained on "
            "plain batched FP64 solves, evaluated on 2000 held-out maps (seeds 100000-101999)")
SUR_GATES = (1e-3, 3e-4, 1e-4, 3e-5)
SUR_SPREADS = (2e-2, 1e-2, 5e-3, 2.5e-3)   # ensemble: largest relative distance of a member from the mean


def run_surrogate_reference(args):
    """The reference's CPU path (the oracle) on held-out surrogate instances, one whole solve per step."""
    from oracle import scattervolume as osv
    from scattersim_b200 import surrogate as sg
    times = []
    for j in range(args.warmup + args.steps):
        m, lam = sg.instance(100000 + j)
        kw = dict(lambda_=float(lam), size=(sg.PERIOD, sg.PERIOD, sg.SLAB), coef=(sg.ORDERS, sg.ORDERS),
                  ex=(1.0, 0.0), ey=(0.0, 0.0), external=True)
        t0 = time.perf_counter()
        osv.solve(np.asarray(m, dtype=np.complex128).reshape(1, 64, 64), osv.Params(**kw), keep=False)
        if j >= args.warmup:
            times.append(time.perf_counter() - t0)
    value = 1.0 / statistics.mean(times)
    line = {"impl": "reference", "metric": SUR_METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * statistics.mean(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": SUR_NAME},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": blas_threads(), "kind": "port",
                             "sample": "one held-out instance per step through the oracle (11x11 orders, one layer, "
                                       "--external)"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_surrogate_ours(args):
    """Train the network on plain solves, then time and score it on held-out maps with the fallback, for a range
    of energy-balance gates.  One step = predicting (with fallback) the 2000 held-out maps."""
    import torch
    from scattersim_b200 import solver
    from scattersim_b200 import surrogate as sg
    torch.cuda.set_device(0)
    ctx = solver.Context(0)
    t0 = time.perf_counter()
    tmaps, tlams, tx = sg.generate(ctx, range(args.train_solves))
    maps, lams, xs = sg.generate(ctx, range(100000, 102000))
    gen_s = time.perf_counter() - t0
    # one network, or an ensemble of networks from different initialisations and shuffles
    surs = [sg.Surrogate(0, max_batch=64, seed=i) for i in range(max(1, args.ensemble))]
    t0 = time.perf_counter()
    ttgt = np.stack([sg.x_to_target(x) for x in tx])
    for i, su in enumerate(surs):
        sg.train(su, tmaps, tlams, ttgt, args.epochs, 64, 1e-3, seed=i)
        su.status()
    train_s = time.perf_counter() - t0
    dm, dl = torch.from_numpy(maps).cuda(), torch.from_numpy(lams).cuda()
    preds = [sg.target_to_x(su.forward(dm, dl).cpu().numpy()) for su in surs]
    pred = np.mean(preds, axis=0)
    err_net = sg.rel_err(pred, xs)
    energy = sg.energy_error(pred, lams)
    sur = surs if len(surs) > 1 else surs[0]
    stream = torch.cuda.current_stream()

    def timed(fn):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        return out, e0.elapsed_time(e1)

    gates = {}
    # energy-balance gates, and with an ensemble also the members' disagreement (loosest first)
    combos = [(tol, None) for tol in SUR_GATES]
    if len(surs) > 1:
        combos = [(tol, sp) for tol in SUR_GATES[:2] for sp in (None,) + SUR_SPREADS]
    for tol, sp in combos:
        for _ in range(args.warmup):
            sg.predict_with_fallback(sur, ctx, maps, lams, tol, sp)
        ms = []
        for _ in range(args.steps):
            (out, bad), t = timed(lambda: sg.predict_with_fallback(sur, ctx, maps, lams, tol, sp))
            ms.append(t)
        err = sg.rel_err(out, xs)
        gates[f"{tol:g}" if sp is None else f"{tol:g}, spread {sp:g}"] = {
            "solves_per_s": len(maps) / (statistics.mean(ms) / 1e3), "fallback_fraction": float(bad.mean()),
            "rel_err": {"median": float(np.median(err)), "p90": float(np.quantile(err, 0.9)),
                        "max": float(err.max())}}
    # the same held-out maps through the batched plain solve alone (the fallback-only method), and the plain
    # per-instance path on a sample
    _, t_fb = timed(lambda: sg.solve_plain(ctx, maps, lams))
    sub = list(range(0, len(maps), 40))
    t_plain = 0.0
    for i in sub:
        d = torch.from_numpy(maps[i].reshape(1, 64, 64).astype(np.complex128)).cuda()
        _, t = timed(lambda: solver.solve(ctx, sg.params_for(float(lams[i])), d, fields=False))
        t_plain += t
    plain = len(sub) / (t_plain / 1e3)
    # headline gate: the fastest whose p90 error with fallback is within 1e-2
    ok = [k for k in gates if gates[k]["rel_err"]["p90"] <= 1e-2]
    head = max(ok, key=lambda k: gates[k]["solves_per_s"]) if ok else list(gates)[-1]
    value = gates[head]["solves_per_s"]
    line = {"metric": SUR_METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": len(maps) / value * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "bf16 network (fp32 accumulate) + f64 fallback",
            "data": "synthetic",
            "config": {"workload": SUR_NAME, "train_solves": args.train_solves, "epochs": args.epochs,
                       "networks": len(surs),
                       "gate": f"|energy balance error| <= {head.split(',')[0]}" +
                               (f", members' relative disagreement <= {head.split('spread ')[1]}"
                                if "spread" in head else "")},
            "paths": {"gates": gates, "network_alone_rel_err": {"median": float(np.median(err_net)),
                                                                "p90": float(np.quantile(err_net, 0.9)),
                                                                "max": float(err_net.max())},
                      "network_energy_error_median": float(np.median(energy)),
                      "fallback_only_batched_fp64": len(maps) / (t_fb / 1e3),
                      "plain_fp64_per_instance": plain,
                      "speedup_vs_plain": value / plain,
                      "speedup_vs_fallback_only": value / (len(maps) / (t_fb / 1e3)),
                      "generate_s": gen_s, "train_s": train_s}}
    print(json.dumps(line), flush=True)
    for su in surs:
        su.close()
    ctx.close()
    return 0


# --------------------------------------------------------------------------- named profiling cases
# python bench.py --case <case> [args]: one configuration at a time, for timing
# and for the ncu commands of the profile summaries.
#
# Cases (seeded synthetic samples, see samples.py):
#   thin          64x64 triangle map, 10x10 um, 1 um slab, lambda 0.5, 11x11 orders
#   volume        128x128x32 sphere volume, 20x20x8 um, lambda 0.6, 10 deg, 21x21 orders
#   volume8       the same geometry with 8 slices
#   small         128x128x4 sphere volume, 11x11 orders (a short QR capture)
#   fp64          measured FP64 throughput: FMA pipe and mma.sync f64
#   sweep [n]     the uneven sweep (first n of 256 instances: 64 wavelengths x 4
#                 angles, 4-16 layer disk stacks, 7..25 orders) in one batched call
#   sweep_mixed [n]  the sweep with the mixed path (int8 tensor-core products, 7
#                    digit slices, where the autotuner finds them faster)
#   sweep_plain [n]  the same instances, one per-instance solve each
#     (sweep cases accept --choices-out FILE to save the GEMM autotuner's table
#      and --choices-in FILE to replay one, e.g. under a profiler)
#   volume31      the sphere volume at 31x31 orders (M = 961, 3844 x 3844 layer
#                 matrices), solved in FP64 and in mixed precision; prints times
#                 and the mixed path's error per stage against the FP64 path
#   fno_train     20 surrogate training steps (batch 64, random maps and targets):
#                 samples/s and the launch mix of the network's kernels
#   gemm          batched complex GEMM throughput at the shapes of the solves
#   gemm_int8     one int8 digit-sliced GEMM shape (1250^3 x 8) at 7 then 4 slices,
#                 twice each (the profiling case of the tcgen05 MMA kernel)
#   gemm_crt [m n k batch reps tiles]  the modular int8 engine (default 1250^3 x 8): time of
#                 the whole product and of its MMA kernel, error against the FP64 tile
#   layer [N]     scatterlayer's default stack (4 layers) under an N x N polar beam
#                 (default 1024: 1,048,576 waves) and a 15-layer stack under a
#                 256 x 256 beam: waves/s of the beam and of the batched layer
#                 solve (bench.py --workload layer adds the host baseline)

D10 = (math.sin(math.radians(10.0)), 0.0, math.cos(math.radians(10.0)))


def case_sample(name):
    from scattersim_b200 import samples
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


def run_case(argv):
    import torch
    from scattersim_b200 import solver
    name = argv[0]
    reps = int(argv[1]) if len(argv) > 1 else 1
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
    if name == "gemm_crt":
        return gemm_crt_case(*[int(a) for a in argv[1:7]])
    if name == "layer":
        return layer_case(int(argv[1]) if len(argv) > 1 else 1024)
    if name in ("sweep", "sweep_plain", "sweep_mixed"):
        count = int(argv[1]) if len(argv) > 1 and not argv[1].startswith("--") else 256
        opt = dict(zip(argv[2::2], argv[3::2])) if len(argv) > 2 else {}
        return sweep_case(name, count, opt.get("--choices-in"), opt.get("--choices-out"))
    smp, kw = case_sample(name)
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
    from scattersim_b200 import solver
    from scattersim_b200._lib import check
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
    from scattersim_b200 import surrogate as sg
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
    from scattersim_b200 import samples, solver
    from scattersim_b200._lib import SC_SWEEP_FP64, SC_SWEEP_MIXED
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
    from scattersim_b200 import solver
    from scattersim_b200._lib import check
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


def gemm_crt_case(m=1250, n=1250, k=1250, batch=8, reps=3, tiles=0):
    """The modular int8 engine on one shape (default 1250^3 x 8, the sweep's largest layer-factor products):
    FP64-equivalent TFLOP/s of the whole product and of its MMA kernel, int8 TOPS, error vs the FP64 tile.
    tiles: 1 = 256 x 256 tiles on CTA pairs, 0 = 128 x 256 tiles on one CTA."""
    import ctypes
    import torch
    from scattersim_b200 import solver
    from scattersim_b200._lib import check
    ctx = solver.Context(0)
    ctx.crt_tiles(tiles)
    A = torch.randn(batch, k, m, dtype=torch.complex128, device="cuda")
    B = torch.randn(batch, n, k, dtype=torch.complex128, device="cuda")
    C = torch.empty(batch, n, m, dtype=torch.complex128, device="cuda")
    R = torch.empty_like(C)
    one = (ctypes.c_double * 2)(1.0, 0.0)
    zero = (ctypes.c_double * 2)(0.0, 0.0)
    args = (ctx.handle, m, n, k, one, ctypes.c_void_p(A.data_ptr()), m, m * k, ctypes.c_void_p(B.data_ptr()), k,
            k * n, zero, ctypes.c_void_p(C.data_ptr()), m, m * n, batch, None)
    check(ctx.lib.sc_zgemm_batched(*(args[:12] + (ctypes.c_void_p(R.data_ptr()),) + args[13:])))
    for _ in range(2):
        check(ctx.lib.sc_zgemm_crt_batched(*args))
    torch.cuda.synchronize()
    ctx.kernel_timing(True)
    for _ in range(reps):
        check(ctx.lib.sc_zgemm_crt_batched(*args))
    st = ctx.kernel_stats_ex()
    ctx.kernel_timing(False)
    err = float((C - R).abs().max() / R.abs().max())
    fl = 8.0 * m * n * k * batch * reps
    print(f"gemm_crt m={m} n={n} k={k} batch={batch} tiles={'256x256 pair' if tiles else '128x256'}: whole product {st['crt_gemm']['ms'] / reps:.3f} ms "
          f"({fl / (st['crt_gemm']['ms'] / 1e3) / 1e12:.1f} FP64-eq TFLOP/s), MMA kernel "
          f"{st['crt']['ms'] / reps:.3f} ms ({st['crt']['int8_ops'] / (st['crt']['ms'] / 1e3) / 1e12:.0f} int8 TOPS, "
          f"{fl / (st['crt']['ms'] / 1e3) / 1e12:.1f} FP64-eq), max error vs FP64 tile {err:.2e}")
    ctx.close()
    return 0


def sweep_case(name, count, choices_in=None, choices_out=None):
    import time
    import torch
    from scattersim_b200 import samples, solver
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

    from scattersim_b200 import layers, solver
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer loop (profiling runs)")
    ap.add_argument("--workload", default="sweep", choices=["sweep", "volume", "layer", "field", "surrogate"])
    ap.add_argument("--train-solves", type=int, default=150000, help="surrogate workload: training solves")
    ap.add_argument("--epochs", type=int, default=30, help="surrogate workload: training epochs")
    ap.add_argument("--ensemble", type=int, default=1,
                    help="surrogate workload: networks trained from different seeds (their mean is the prediction; "
                         "with 2 or more, a sample whose members disagree also falls back)")
    ap.add_argument("--case", nargs=argparse.REMAINDER, help="run one named profiling case instead")
    args = ap.parse_args()
    if args.case:
        return run_case(args.case)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "sweep":
        return run_sweep_ours(args)
    if args.workload == "layer":
        return run_layer_ours(args)
    if args.workload == "field":
        return run_field_ours(args)
    if args.workload == "surrogate":
        return run_surrogate_ours(args)
    return run_volume_ours(args)


if __name__ == "__main__":
    sys.exit(main())
