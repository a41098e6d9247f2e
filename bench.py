#!/usr/bin/env python
"""Benchmark: scattervolume solves/s on B200.

Workload (default): the plain 3-D volume -- a 128x128x32-voxel sphere volume
over 20x20x8 um (seeded), 32 layers, lambda = 0.6 um, 10 deg incidence,
x-polarised, 21x21 Fourier orders (M = 441, 1764 x 1764 layer matrices),
solved in FP64 with the interior mode fields (the reference's default, Pz on).
One step = one full solve of one instance, sample resident in HBM.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun each rank solves its own seeded instance (weak scaling, no
data-path collective); timing is on the device, max over ranks.
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


def run_ours(args):
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer loop (profiling runs)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
