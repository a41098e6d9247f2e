"""Learned surrogate of the thin-volume solve, with the plain solve as fallback.

    python -m scattersim_b200.surrogate run [--train N] [--test N] [--epochs E] [--out DIR]

Workload (seeded): 64x64 index maps over a 10x10 um period holding 1-4 random
disks and/or triangles with n in [1.0, 1.6] (background 1.0), a 1 um slab,
lambda in [0.4, 0.8] um, normal incidence, x-polarised, 11x11 orders.  The
batched FP64 solve (sc_sweep_solve) generates the targets -- the R/T vector x
of ScatterVolume.cpp:739 -- for training seeds 0.. and held-out seeds
100000..; the network (sc_fno_*) is trained on the GPU by the library's own
BF16/FP32 kernels.  At inference every prediction is checked for energy
balance (|sum |R|^2 Sz_top + |T|^2 Sz_bot - 1| <= 1e-3 for the unit incident
flux of this workload); a sample that fails is solved by the plain solve.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import time

import numpy as np
import torch

from . import _lib, solver
from ._lib import check

PERIOD = 10.0
SLAB = 1.0
ORDERS = 11
NORD = ORDERS * ORDERS
NOUT = 6 * NORD * 2
ENERGY_TOL = 1e-3


def surrogate_map(rng, n: int = 64, period: float = PERIOD) -> np.ndarray:
    """(n, n) real index map: 1-4 disks (r 0.5-2.5 um) and/or triangles, n in [1.0, 1.6]."""
    c = (np.arange(n) + 0.5) * (period / n)
    Y, X = np.meshgrid(c, c, indexing="ij")
    m = np.ones((n, n))
    for _ in range(int(rng.integers(1, 5))):
        val = rng.uniform(1.0, 1.6)
        if rng.uniform() < 0.5:
            cc = rng.uniform(0, period, 2)
            r = rng.uniform(0.5, 2.5)
            m[(X - cc[0]) ** 2 + (Y - cc[1]) ** 2 <= r * r] = val
        else:
            v = rng.uniform(0, period, (3, 2))

            def side(a, b):
                return (X - a[0]) * (b[1] - a[1]) - (Y - a[1]) * (b[0] - a[0])
            s0, s1, s2 = side(v[0], v[1]), side(v[1], v[2]), side(v[2], v[0])
            inside = ((s0 >= 0) & (s1 >= 0) & (s2 >= 0)) | ((s0 <= 0) & (s1 <= 0) & (s2 <= 0))
            m[inside] = val
    return m


def instance(seed: int):
    """(map (64, 64) float64, wavelength) of one seeded surrogate instance."""
    rng = np.random.default_rng(seed)
    lam = float(rng.uniform(0.4, 0.8))
    return surrogate_map(rng), lam


def params_for(lam: float):
    return solver.make_params(lambda_=lam, size=(PERIOD, PERIOD, SLAB), coef=(ORDERS, ORDERS), ex=(1.0, 0.0),
                              ey=(0.0, 0.0), external=True)


def x_to_target(x: np.ndarray) -> np.ndarray:
    """complex (726,) R/T vector -> 1452 floats (re, im interleaved)."""
    return np.stack([x.real, x.imag], axis=-1).reshape(-1).astype(np.float32)


def target_to_x(t) -> np.ndarray:
    t = np.asarray(t, np.float64).reshape(-1, 6 * NORD, 2)
    return t[..., 0] + 1j * t[..., 1]


def solve_plain(ctx, maps: np.ndarray, lams, chunk: int = 1024, precision: int = _lib.SC_SWEEP_FP64):
    """R/T vectors (N, 726) complex128 of maps (N, 64, 64) by the batched plain solve."""
    out = []
    for i0 in range(0, len(maps), chunk):
        ms = maps[i0:i0 + chunk]
        ls = lams[i0:i0 + chunk]
        params = [params_for(float(l)) for l in ls]
        smp = [torch.from_numpy(np.ascontiguousarray(m.reshape(1, 64, 64).astype(np.complex128))).cuda() for m in ms]
        res = solver.sweep(ctx, params, smp, precision=precision)
        out.extend(x.cpu().numpy() for x in res.x)
    return np.stack(out)


def generate(ctx, seeds):
    """Maps and wavelengths of the seeded instances (float32, as the network reads
    them) and the plain solve's R/T vectors of exactly those float32 inputs."""
    seeds = list(seeds)
    maps = np.empty((len(seeds), 64, 64), dtype=np.float32)
    lams = np.empty(len(seeds), dtype=np.float32)
    for i, s in enumerate(seeds):
        m, lam = instance(int(s))
        maps[i] = m
        lams[i] = lam
    x = solve_plain(ctx, maps, lams)
    return maps, lams, x


def energy_error(x: np.ndarray, lams) -> np.ndarray:
    """|sum_orders |R|^2 Re Sz_top + |T|^2 Re Sz_bot - 1| per sample (unit incident flux).

    Sx = p lambda / period, Sy = q lambda / period at order index j = i + 11 jj
    (q = i - 5, p = jj - 5; the column-major order index of the solve)."""
    x = np.asarray(x).reshape(-1, 6, NORD)
    j = np.arange(NORD)
    q = j % ORDERS - ORDERS // 2
    p = j // ORDERS - ORDERS // 2
    lam = np.asarray(lams, np.float64)[:, None]
    sz = np.sqrt((1.0 - (p[None] * lam / PERIOD) ** 2 - (q[None] * lam / PERIOD) ** 2).astype(np.complex128)).real
    R = (np.abs(x[:, 0:3]) ** 2).sum(1)
    T = (np.abs(x[:, 3:6]) ** 2).sum(1)
    return np.abs((R * sz).sum(1) + (T * sz).sum(1) - 1.0)


def rel_err(a, b) -> np.ndarray:
    a = np.asarray(a).reshape(len(b), -1)
    b = np.asarray(b).reshape(len(b), -1)
    return np.linalg.norm(a - b, axis=1) / np.linalg.norm(b, axis=1)


class Surrogate:
    """The library's FNO (sc_fno_*) with torch tensors as device buffers."""

    def __init__(self, device: int = 0, max_batch: int = 64, seed: int = 0):
        self.lib = _lib.load()
        h = ctypes.c_void_p()
        check(self.lib.sc_fno_create(ctypes.byref(h), device, max_batch, seed))
        self.h = h
        self.device = torch.device("cuda", device)
        self.max_batch = max_batch
        n = ctypes.c_longlong(0)
        check(self.lib.sc_fno_param_count(self.h, ctypes.byref(n)))
        self.n_params = n.value

    def close(self):
        if self.h is not None and self.h.value:
            self.lib.sc_fno_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def _p(t):
        return ctypes.c_void_p(t.data_ptr())

    def _buf(self, t, shape, name: str) -> torch.Tensor:
        """`t` as a contiguous float32 tensor on the network's device, after checking its shape: the library
        reads as many floats as the batch implies from a bare pointer, so a short buffer must not reach it."""
        t = torch.as_tensor(t)
        if tuple(t.shape) != tuple(shape):
            raise ValueError(f"surrogate: {name} has shape {tuple(t.shape)}, expected {tuple(shape)}")
        return t.to(device=self.device, dtype=torch.float32).contiguous()

    def _batch(self, maps, lams, target=None):
        """(batch, [maps, lams(, target)]) checked and placed for one library call."""
        maps = torch.as_tensor(maps)
        B = int(maps.shape[0]) if maps.dim() else 0
        bufs = [self._buf(maps, (B, 64, 64), "maps"), self._buf(lams, (B,), "lams")]
        if target is not None:
            bufs.append(self._buf(target, (B, NOUT), "target"))
        return B, bufs

    def status(self):
        """Synchronise and raise if a tensor-core GEMM of this network timed out since the last check."""
        check(self.lib.sc_fno_status(self.h))

    def get_params(self) -> torch.Tensor:
        t = torch.empty(self.n_params, dtype=torch.float32, device=self.device)
        check(self.lib.sc_fno_params(self.h, self._p(t), 0, None))
        torch.cuda.synchronize()
        return t

    def set_params(self, t):
        t = self._buf(torch.as_tensor(t).reshape(-1), (self.n_params,), "parameters")
        check(self.lib.sc_fno_params(self.h, self._p(t), 1, None))
        torch.cuda.synchronize()

    def forward(self, maps: torch.Tensor, lams: torch.Tensor) -> torch.Tensor:
        B, (maps, lams) = self._batch(maps, lams)
        out = torch.empty((B, NOUT), dtype=torch.float32, device=self.device)
        for i0 in range(0, B, self.max_batch):
            m = maps[i0:i0 + self.max_batch].contiguous()
            l = lams[i0:i0 + self.max_batch].contiguous()
            check(self.lib.sc_fno_forward(self.h, self._p(m), self._p(l), m.shape[0], self._p(out[i0:]), None))
        return out

    def loss_grad(self, maps, lams, target):
        B, (maps, lams, target) = self._batch(maps, lams, target)
        loss = torch.empty(B, dtype=torch.float32, device=self.device)
        grad = torch.empty(self.n_params, dtype=torch.float32, device=self.device)
        check(self.lib.sc_fno_loss_grad(self.h, self._p(maps), self._p(lams), self._p(target), B, self._p(loss),
                                        self._p(grad), None))
        torch.cuda.synchronize()
        return loss, grad

    def train_step(self, maps, lams, target, lr: float) -> torch.Tensor:
        B, (maps, lams, target) = self._batch(maps, lams, target)
        loss = torch.empty(B, dtype=torch.float32, device=self.device)
        check(self.lib.sc_fno_train_step(self.h, self._p(maps), self._p(lams), self._p(target), B, float(lr),
                                         self._p(loss), None))
        return loss


def train(sur: Surrogate, maps, lams, targets, epochs: int, batch: int = 64, lr: float = 1e-3, seed: int = 0,
          log=None):
    """Adam with a cosine rate schedule over `epochs` passes of shuffled batches."""
    dev = sur.device
    dm = torch.as_tensor(np.ascontiguousarray(maps, dtype=np.float32), device=dev)
    dl = torch.as_tensor(np.ascontiguousarray(lams, dtype=np.float32), device=dev)
    dt = torch.as_tensor(np.ascontiguousarray(targets, dtype=np.float32), device=dev)
    n = len(maps)
    rng = np.random.default_rng(seed)
    steps = epochs * (n // batch)
    step = 0
    hist = []
    for ep in range(epochs):
        perm = torch.from_numpy(rng.permutation(n)).to(dev)
        # the loss is summed on the device: reading it back every step would
        # stall the launch queue once per step
        tot = torch.zeros((), dtype=torch.float32, device=dev)
        for i0 in range(0, n - batch + 1, batch):
            idx = perm[i0:i0 + batch]
            rate = lr * 0.5 * (1.0 + math.cos(math.pi * step / max(steps, 1)))
            loss = sur.train_step(dm[idx].contiguous(), dl[idx].contiguous(), dt[idx].contiguous(), rate)
            tot += loss.mean()
            step += 1
        hist.append(float(tot) / max(1, n // batch))
        if log:
            log(f"epoch {ep}: train loss {hist[-1]:.3e}")
    torch.cuda.synchronize()
    return hist


def predict_with_fallback(sur, ctx, maps, lams, tol: float = ENERGY_TOL, spread: float | None = None):
    """Surrogate R/T (N, 726) complex, with the plain solve wherever energy balance fails.

    `sur` is one Surrogate or a list of them (an ensemble trained from different seeds): the prediction is the
    members' mean, and with `spread` a sample whose members disagree (the largest relative distance of a member
    from the mean) by more than `spread` falls back as well."""
    members = list(sur) if isinstance(sur, (list, tuple)) else [sur]
    if not members:
        raise ValueError("predict_with_fallback: no network given")
    dm = torch.as_tensor(np.ascontiguousarray(maps, dtype=np.float32), device=members[0].device)
    dl = torch.as_tensor(np.ascontiguousarray(lams, dtype=np.float32), device=members[0].device)
    preds = [target_to_x(m.forward(dm, dl).cpu().numpy()) for m in members]
    pred = np.mean(preds, axis=0) if len(preds) > 1 else preds[0]
    bad = energy_error(pred, lams) > tol
    if spread is not None and len(preds) > 1:
        dis = np.max([rel_err(q, pred) for q in preds], axis=0)
        bad |= dis > spread
    if bad.any():
        pred[bad] = solve_plain(ctx, np.asarray(maps)[bad], np.asarray(lams)[bad])
    return pred, bad


def run(args):
    ctx = solver.Context(0)
    log = print
    t0 = time.perf_counter()
    tr = generate(ctx, range(args.train))
    te = generate(ctx, range(100000, 100000 + args.test))
    torch.cuda.synchronize()
    log(f"generated {args.train} + {args.test} solves in {time.perf_counter() - t0:.1f} s")
    tmaps, tlams, tx = tr
    targets = np.stack([x_to_target(x) for x in tx])
    sur = Surrogate(0, max_batch=args.batch, seed=args.seed)
    t0 = time.perf_counter()
    hist = train(sur, tmaps, tlams, targets, args.epochs, args.batch, args.lr, log=log)
    t_train = time.perf_counter() - t0
    maps, lams, xs = te
    # held-out error of the network alone, and of the network with fallback
    dm = torch.from_numpy(maps).cuda()
    dl = torch.from_numpy(lams).cuda()
    pred = target_to_x(sur.forward(dm, dl).cpu().numpy())
    err_net = rel_err(pred, xs)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    out, bad = predict_with_fallback(sur, ctx, maps, lams)
    torch.cuda.synchronize()
    t_sur = time.perf_counter() - t0
    err_fb = rel_err(out, xs)
    # the plain per-instance path on a sample of the held-out set
    sub = range(0, len(maps), max(1, len(maps) // 64))
    t0 = time.perf_counter()
    for i in sub:
        solver.solve(ctx, params_for(float(lams[i])),
                     torch.from_numpy(maps[i].reshape(1, 64, 64).astype(np.complex128)).cuda(), fields=False)
    torch.cuda.synchronize()
    t_plain = (time.perf_counter() - t0) / len(sub)
    res = {"train": args.train, "test": args.test, "epochs": args.epochs, "train_s": t_train,
           "final_train_loss": hist[-1],
           "net_rel_err": {"median": float(np.median(err_net)), "p90": float(np.quantile(err_net, 0.9)),
                           "max": float(err_net.max())},
           "fallback_fraction": float(bad.mean()),
           "with_fallback_rel_err": {"median": float(np.median(err_fb)), "p90": float(np.quantile(err_fb, 0.9)),
                                     "max": float(err_fb.max())},
           "surrogate_with_fallback_solves_per_s": len(maps) / t_sur,
           "plain_per_instance_solves_per_s": 1.0 / t_plain,
           "speedup_vs_plain": (len(maps) / t_sur) * t_plain}
    log(json.dumps(res))
    if args.out:
        os.makedirs(args.out, exist_ok=True)
        np.save(os.path.join(args.out, "fno_params.npy"), sur.get_params().cpu().numpy())
        with open(os.path.join(args.out, "surrogate.json"), "w") as f:
            json.dump(res, f, indent=1)
    sur.close()
    ctx.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("cmd", choices=["run"])
    ap.add_argument("--train", type=int, default=20000)
    ap.add_argument("--test", type=int, default=2000)
    ap.add_argument("--epochs", type=int, default=30)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--out", default="")
    return run(ap.parse_args())


if __name__ == "__main__":
    raise SystemExit(main())
