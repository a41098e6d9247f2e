"""ScatterVolume: the scattervolume solve through the C ABI.

Mirrors the reference's command-line surface (ScatterVolume.cpp:511-529:
--sample --lambda --direction --ex --ey --ez --n --kappa --size --z --coef
--psf --external --npz) as keyword arguments with the same defaults.  Device
buffers are torch tensors (plumbing only); every computation runs in
libscattersim_b200.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import VolumeDims, VolumeParams, check


def _stream_ptr(stream=None):
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


def _checked(ctx, t, shape, name: str, dtype=torch.complex128) -> torch.Tensor:
    """`t` made contiguous after checking its type, its device (the context's) and its shape (None: any): the
    library reads as many elements as the sizes imply from a bare pointer, so a short buffer must not reach it."""
    if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != dtype:
        raise TypeError(f"{name} must be a {dtype} CUDA tensor")
    if t.device.index != ctx.device:
        raise ValueError(f"{name} is on {t.device}, the context on cuda:{ctx.device}")
    if shape is not None and tuple(t.shape) != tuple(shape):
        raise ValueError(f"{name} has shape {tuple(t.shape)}, expected {tuple(shape)}")
    return t.contiguous()


class Context:
    """One sc_context per GPU (pooled device workspace)."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        self.device = device
        h = ctypes.c_void_p()
        check(self.lib.sc_create(ctypes.byref(h), device))
        self.handle = h

    def close(self):
        if self.handle is not None and self.handle.value:
            self.lib.sc_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def launches(self) -> int:
        return int(self.lib.sc_launch_count(self.handle))

    def stage_ms(self):
        """Device ms of the last solve per stage, plus the QR kernel alone and the total."""
        out = (ctypes.c_double * 8)()
        check(self.lib.sc_volume_stage_ms(self.handle, out))
        return dict(zip(("fft", "assemble", "eig", "chain", "boundary", "interior", "qr", "total"), list(out)))

    def qr_stats(self, count: int):
        """Per matrix of the last eigensolve: sweeps and SM cycles of the QR phases."""
        out = (ctypes.c_longlong * (8 * count))()
        check(self.lib.sc_qr_stats(self.handle, out, count))
        keys = ("sweeps", "shifts", "chase", "far_right", "far_rows", "small", "unused", "total")
        return [dict(zip(keys, out[8 * i:8 * i + 8])) for i in range(count)]

    def set_precision(self, precision: int):
        """Precision code (SC_SWEEP_*) of the products of later solve() calls."""
        check(self.lib.sc_volume_precision(self.handle, int(precision)))

    def kernel_timing(self, on: bool = True):
        """Start (clearing the record) or stop per-launch timing of the engine's GEMM kernels."""
        check(self.lib.sc_kernel_timing(self.handle, int(on)))

    def kernel_stats(self):
        """{'dmma': {...}, 'int8': {...}}: launches, ms, FP64-equivalent flops, int8 ops."""
        out = (ctypes.c_double * 8)()
        check(self.lib.sc_kernel_stats(self.handle, out))
        keys = ("launches", "ms", "flops", "int8_ops")
        return {"dmma": dict(zip(keys, out[0:4])), "int8": dict(zip(keys, out[4:8]))}

    def kernel_stats_ex(self):
        """Per kernel class: 'dmma' FP64 tiles, 'int8' digit-sliced MMA kernel, 'crt' modular MMA kernel,
        'crt_gemm' whole modular-engine products; each {launches, ms, flops, int8_ops}."""
        out = (ctypes.c_double * 16)()
        check(self.lib.sc_kernel_stats_ex(self.handle, out, 4))
        keys = ("launches", "ms", "flops", "int8_ops")
        return {name: dict(zip(keys, out[4 * i:4 * i + 4])) for i, name in
                enumerate(("dmma", "int8", "crt", "crt_gemm"))}

    def gemm_choices(self):
        """The autotuner's table: list of (m, n, k, batch, slices, variant)."""
        n = ctypes.c_int(0)
        check(self.lib.sc_gemm_choices_get(self.handle, None, 0, ctypes.byref(n)))
        buf = (ctypes.c_int * (6 * max(n.value, 1)))()
        check(self.lib.sc_gemm_choices_get(self.handle, buf, n.value, ctypes.byref(n)))
        return [tuple(buf[6 * i:6 * i + 6]) for i in range(n.value)]

    def set_gemm_choices(self, table):
        flat = [int(v) for rec in table for v in rec]
        buf = (ctypes.c_int * max(len(flat), 1))(*flat)
        check(self.lib.sc_gemm_choices_set(self.handle, buf, len(table)))

    def int8_peak_tops(self) -> float:
        """Measured int8 tcgen05 MMA throughput (TOPS), operands resident in shared memory."""
        v = ctypes.c_double(0.0)
        check(self.lib.sc_int8_peak_probe(self.handle, ctypes.byref(v)))
        return v.value

    def crt_tiles(self, mode: int) -> None:
        """Modular engine's MMA tiles: 0 = 128 x 256 on one CTA (default), 1 = 256 x 256 on CTA pairs."""
        check(self.lib.sc_crt_tiles_set(self.handle, int(mode)))

    def fp64_peak_tflops(self, tensor: bool = False) -> float:
        """Measured FP64 throughput: FMA pipe, or mma.sync f64 with tensor=True."""
        v = ctypes.c_double(0.0)
        f = self.lib.sc_fp64_dmma_probe if tensor else self.lib.sc_fp64_peak_probe
        check(f(self.handle, ctypes.byref(v)))
        return v.value


def make_params(lambda_=1.0, direction=(0, 0, 1), ex=(0, 0), ey=(1, 0), ez=(0, 0), n=(1, 1), kappa=0.0,
                size=(10, 10, 2), z=0.0, coef=(), psf=False, external=False, npz=False) -> VolumeParams:
    """sc_volume_params with the reference's defaults (ScatterVolume.cpp:511-529)."""
    p = VolumeParams()
    p.lambda_ = float(lambda_)
    for i in range(3):
        p.direction[i] = float(direction[i])
        p.size[i] = float(size[i])
    for i in range(2):
        p.ex[i], p.ey[i], p.ez[i], p.n[i] = float(ex[i]), float(ey[i]), float(ez[i]), float(n[i])
    kap = kappa[0] if isinstance(kappa, (tuple, list)) else kappa
    p.kappa = float(kap)
    p.z = float(z)
    coef = tuple(coef)
    p.ncoef = len(coef)
    for i, c in enumerate(coef[:2]):
        p.coef[i] = int(c)
    p.psf, p.external, p.npz = int(psf), int(external), int(npz)
    return p


def plan(params: VolumeParams, shape) -> VolumeDims:
    Z, S1, S2 = shape
    d = VolumeDims()
    check(_lib.load().sc_volume_plan(ctypes.byref(params), Z, S1, S2, ctypes.byref(d)))
    return d


@dataclass
class VolumeSolution:
    dims: VolumeDims
    shape: tuple
    x: torch.Tensor          # (6 MF,) complex128: [R_x R_y R_z T_x T_y T_z]
    evl: torch.Tensor        # (Z, 4 MF)
    Qc: torch.Tensor         # (Z, 2MF, 3MF) -> column-major 3MF x 2MF blocks
    Qh: torch.Tensor


def solve(ctx: Context, params: VolumeParams, sample: torch.Tensor, fields: bool = True, stream=None):
    """One scattervolume solve of a device-resident (Z, S1, S2) complex128 sample."""
    if sample.dim() == 2:
        sample = sample.unsqueeze(0)
    sample = _checked(ctx, sample, None, "sample")
    shape = tuple(sample.shape)
    d = plan(params, shape)
    MF, Z = d.MF, shape[0]
    dev = sample.device
    x = torch.empty(6 * MF, dtype=torch.complex128, device=dev)
    evl = torch.empty((Z, 4 * MF), dtype=torch.complex128, device=dev)
    want = fields and not params.external
    Qc = torch.empty((Z, 2 * MF, 3 * MF), dtype=torch.complex128, device=dev) if want else None
    Qh = torch.empty((Z, 2 * MF, 3 * MF), dtype=torch.complex128, device=dev) if want else None
    info = ctypes.c_int(0)
    check(ctx.lib.sc_volume_solve(ctx.handle, ctypes.byref(params), _ptr(sample), *shape, _ptr(x), _ptr(evl),
                                  _ptr(Qc), _ptr(Qh), ctypes.byref(info), _stream_ptr(stream)))
    return VolumeSolution(d, shape, x, evl, Qc, Qh)


def chain_block(ctx: Context, params: VolumeParams, sample: torch.Tensor, layer_begin: int, layer_end: int,
                stream=None):
    """(P, GD0): the ordered transfer product of layers [begin, end) (4MF x 4MF, column-major storage in a
    (4MF, 4MF) tensor read as its transpose) and GD_0 for the block that starts at layer 0 (else None)."""
    if sample.dim() == 2:
        sample = sample.unsqueeze(0)
    sample = _checked(ctx, sample, None, "sample")
    shape = tuple(sample.shape)
    d = plan(params, shape)
    n4 = 4 * d.MF
    P = torch.empty((n4, n4), dtype=torch.complex128, device=sample.device)
    GD0 = torch.empty((n4, n4), dtype=torch.complex128, device=sample.device) if layer_begin == 0 else None
    info = ctypes.c_int(0)
    check(ctx.lib.sc_volume_chain_block(ctx.handle, ctypes.byref(params), _ptr(sample), *shape, int(layer_begin),
                                        int(layer_end), _ptr(P), _ptr(GD0), ctypes.byref(info), _stream_ptr(stream)))
    return P, GD0


def boundary_solve(ctx: Context, params: VolumeParams, shape, Gc_static: torch.Tensor, GD0: torch.Tensor,
                   stream=None) -> torch.Tensor:
    """x = [R; T] (6 MF) from the whole chain and GD_0 (storage as chain_block returns them)."""
    shape = tuple(shape)
    if len(shape) == 2:
        shape = (1,) + shape
    d = plan(params, shape)
    n4 = 4 * d.MF
    Gc_static = _checked(ctx, Gc_static, (n4, n4), "Gc_static")
    GD0 = _checked(ctx, GD0, (n4, n4), "GD0")
    x = torch.empty(6 * d.MF, dtype=torch.complex128, device=Gc_static.device)
    info = ctypes.c_int(0)
    check(ctx.lib.sc_volume_boundary_solve(ctx.handle, ctypes.byref(params), *shape, _ptr(Gc_static), _ptr(GD0),
                                           _ptr(x), ctypes.byref(info), _stream_ptr(stream)))
    return x


def colmajor_matmul(ctx: Context, A: torch.Tensor, B: torch.Tensor, stream=None) -> torch.Tensor:
    """A B for square matrices held in column-major storage (as chain_block returns them), on the FP64 tile."""
    n = A.shape[0] if A.dim() == 2 else -1
    A = _checked(ctx, A, (n, n), "A")
    B = _checked(ctx, B, (n, n), "B")
    C = torch.empty_like(A)
    one = (ctypes.c_double * 2)(1.0, 0.0)
    zero = (ctypes.c_double * 2)(0.0, 0.0)
    check(ctx.lib.sc_zgemm_batched(ctx.handle, n, n, n, one, _ptr(A), n, n * n, _ptr(B), n, n * n, zero, _ptr(C), n,
                                   n * n, 1, _stream_ptr(stream)))
    return C


def split_solve(ctx: Context, params: VolumeParams, sample: torch.Tensor, dist=None, stream=None) -> torch.Tensor:
    """R/T of one volume solved with its layers split over the ranks of `dist` (one exchange of chain blocks)."""
    from . import layersplit
    if sample.dim() == 2:
        sample = sample.unsqueeze(0)
    shape = tuple(sample.shape)
    d = plan(params, shape)
    return layersplit.split_solve(
        shape[0], lambda lb, le: chain_block(ctx, params, sample, lb, le, stream),
        lambda a, b: colmajor_matmul(ctx, a, b, stream),
        lambda g, gd: boundary_solve(ctx, params, shape, g, gd, stream), 6 * d.MF, dist, sample.device)


@dataclass
class WaveTable:
    E0: torch.Tensor         # (nw, 3) complex128
    k: torch.Tensor          # (nw, 3) complex128
    begin: np.ndarray        # (Z + 2,)
    end: np.ndarray
    z_layers: np.ndarray     # (Z + 1,)


def waves(ctx: Context, params: VolumeParams, sol: VolumeSolution, ez_mode: int = 0, stream=None) -> WaveTable:
    """The CoupledWaveStructure wave list of a solution, on the device (cw_unpack order)."""
    Z, S1, S2 = sol.shape
    nw = ctypes.c_longlong(0)
    begin = (ctypes.c_int * (Z + 2))()
    end = (ctypes.c_int * (Z + 2))()
    zl = (ctypes.c_double * (Z + 1))()
    check(ctx.lib.sc_volume_waves(ctx.handle, ctypes.byref(params), Z, S1, S2, None, None, None, None, ez_mode,
                                  ctypes.byref(nw), begin, end, zl, None, None, None))
    E0 = torch.empty((nw.value, 3), dtype=torch.complex128, device=sol.x.device)
    K = torch.empty((nw.value, 3), dtype=torch.complex128, device=sol.x.device)
    check(ctx.lib.sc_volume_waves(ctx.handle, ctypes.byref(params), Z, S1, S2, _ptr(sol.x), _ptr(sol.evl),
                                  _ptr(sol.Qc), _ptr(sol.Qh), ez_mode, ctypes.byref(nw), begin, end, zl, _ptr(E0),
                                  _ptr(K), _stream_ptr(stream)))
    return WaveTable(E0, K, np.array(begin[:]), np.array(end[:]), np.array(zl[:]))


def evaluate(ctx: Context, E0: torch.Tensor, K: torch.Tensor, z_layers, begin, end, points: torch.Tensor,
             zeps: float = 0.001, precision: int = 0, stream=None) -> torch.Tensor:
    """E at (P, 3) float64 device points: the gpuEvaluator sum (gpuEvaluator.cu:28-68)."""
    layers = len(z_layers)
    if len(begin) < layers + 1 or len(end) < layers + 1:
        raise ValueError(f"begin / end need {layers + 1} region bounds")
    zl = (ctypes.c_double * max(layers, 1))(*list(z_layers))
    b = (ctypes.c_int * (layers + 1))(*[int(v) for v in begin[:layers + 1]])
    e = (ctypes.c_int * (layers + 1))(*[int(v) for v in end[:layers + 1]])
    nw = E0.shape[0] if E0.dim() == 2 else -1
    E0 = _checked(ctx, E0, (nw, 3), "E0")
    K = _checked(ctx, K, (nw, 3), "K")
    if not isinstance(points, torch.Tensor) or not points.is_floating_point() or points.dim() != 2 \
            or points.shape[1] != 3:
        raise ValueError("points must be a (P, 3) floating-point tensor")
    points = _checked(ctx, points.to(torch.float64), None, "points", torch.float64)
    out = torch.empty((points.shape[0], 3), dtype=torch.complex128, device=points.device)
    check(ctx.lib.sc_cw_evaluate(ctx.handle, _ptr(E0), _ptr(K), int(E0.shape[0]), zl, b,
                                 e, layers, float(zeps), _ptr(points), int(points.shape[0]), _ptr(out),
                                 int(precision), _stream_ptr(stream)))
    return out


def field_grid(ctx: Context, params: VolumeParams, sol: VolumeSolution, origin, step, counts, ez_mode: int = 0,
               zeps: float = 0.001, precision: int = 0, stream=None) -> torch.Tensor:
    """E on the grid origin + (i, j, b) * step, counts = (Nx, Ny, Nz): a (Nz, Ny, Nx, 3) complex tensor
    (complex128, or complex64 with precision=1) -- the evaluator sum over the solution's waves, factorised."""
    Z, S1, S2 = sol.shape
    nx, ny, nz = (int(c) for c in counts)
    dt = torch.complex128 if precision == 0 else torch.complex64
    out = torch.empty((nz, ny, nx, 3), dtype=dt, device=sol.x.device)
    o = (ctypes.c_double * 3)(*[float(v) for v in origin])
    s = (ctypes.c_double * 3)(*[float(v) for v in step])
    c = (ctypes.c_int * 3)(nx, ny, nz)
    check(ctx.lib.sc_volume_field_grid(ctx.handle, ctypes.byref(params), Z, S1, S2, _ptr(sol.x), _ptr(sol.evl),
                                       _ptr(sol.Qc), _ptr(sol.Qh), int(ez_mode), o, s, c, float(zeps), _ptr(out),
                                       int(precision), _stream_ptr(stream)))
    return out


def empty_solution(ctx: Context, params: VolumeParams, shape, fields: bool = True) -> VolumeSolution:
    """A VolumeSolution of the planned shapes with uninitialised tensors on the context's device: the buffers a
    rank receives a solution into."""
    shape = tuple(shape)
    if len(shape) == 2:
        shape = (1,) + shape
    d = plan(params, shape)
    MF, Z = d.MF, shape[0]
    dev = torch.device("cuda", ctx.device)
    want = fields and not params.external

    def z(*s):
        return torch.empty(s, dtype=torch.complex128, device=dev)
    return VolumeSolution(d, shape, z(6 * MF), z(Z, 4 * MF), z(Z, 2 * MF, 3 * MF) if want else None,
                          z(Z, 2 * MF, 3 * MF) if want else None)


def split_field_grid(ctx: Context, params: VolumeParams, sol: VolumeSolution, origin, step, counts, dist=None,
                     gather: bool = True, ez_mode: int = 0, zeps: float = 0.001, precision: int = 0, stream=None):
    """field_grid with the grid's z-planes split over the ranks of `dist` (contiguous slabs).

    Rank 0's solution is broadcast once to the other ranks (which pass a solution of the same shapes, for
    example from empty_solution); each rank evaluates its slab of planes; with gather every rank returns the
    whole (Nz, Ny, Nx, 3) grid, without it (its slab or None, (first plane, end plane)).
    """
    from . import fieldsplit
    if dist is not None and dist.is_initialized() and dist.get_world_size() > 1:
        fieldsplit.broadcast_tensors([sol.x, sol.evl, sol.Qc, sol.Qh], dist, src=0)
    o = [float(v) for v in origin]
    st = [float(v) for v in step]
    nx, ny, nz = (int(c) for c in counts)

    def slab(b, e):
        return field_grid(ctx, params, sol, (o[0], o[1], o[2] + b * st[2]), st, (nx, ny, e - b), ez_mode, zeps,
                          precision, stream)
    dt = torch.complex128 if precision == 0 else torch.complex64
    return fieldsplit.split_grid(slab, (nx, ny, nz), dist, torch.device("cuda", ctx.device), dt, gather)


@dataclass
class SweepResult:
    x: list                  # per instance: (6 MF,) complex128 device tensor [R; T]
    status: list             # per instance sc_status
    dims: list               # per instance VolumeDims


def sweep(ctx: Context, params, samples, precision: int = _lib.SC_SWEEP_FP64, stream=None,
          raise_on_error: bool = True) -> SweepResult:
    """A batched sweep of independent R/T solves: sc_sweep_solve over device-resident samples.

    params: sequence of VolumeParams; samples: sequence of (Z, S1, S2) (or (S1, S2))
    complex128 CUDA tensors.  Instances may differ in every parameter.
    """
    n = len(params)
    if len(samples) != n:
        raise ValueError("params and samples differ in length")
    smp = []
    for i, t in enumerate(samples):
        if isinstance(t, torch.Tensor) and t.dim() == 2:
            t = t.unsqueeze(0)
        smp.append(_checked(ctx, t, None, f"samples[{i}]"))
    dims = [plan(p, tuple(t.shape)) for p, t in zip(params, smp)]
    xs = [torch.empty(6 * d.MF, dtype=torch.complex128, device=t.device) for d, t in zip(dims, smp)]
    P = (VolumeParams * max(n, 1))(*params)
    S = (ctypes.c_void_p * max(n, 1))(*[t.data_ptr() for t in smp])
    Z = (ctypes.c_int * max(n, 1))(*[t.shape[0] for t in smp])
    S1 = (ctypes.c_int * max(n, 1))(*[t.shape[1] for t in smp])
    S2 = (ctypes.c_int * max(n, 1))(*[t.shape[2] for t in smp])
    X = (ctypes.c_void_p * max(n, 1))(*[x.data_ptr() for x in xs])
    st = (ctypes.c_int * max(n, 1))()
    rc = ctx.lib.sc_sweep_solve(ctx.handle, n, P, S, Z, S1, S2, X, int(precision), st, _stream_ptr(stream))
    if raise_on_error:
        check(rc)
    return SweepResult(xs, list(st[:n]), dims)


def eigensolve(ctx: Context, A: torch.Tensor, stream=None):
    """Batched eigenvalues / right eigenvectors of (B, n, n) complex128 matrices (row-major torch view)."""
    if A.dim() == 2:
        A = A.unsqueeze(0)
    if A.dim() != 3 or A.shape[1] != A.shape[2]:
        raise ValueError(f"A must be (B, n, n) square matrices, got {tuple(A.shape)}")
    A = _checked(ctx, A, None, "A")
    B, n, _ = A.shape
    # C ABI is column-major: pass A^T's storage, i.e. the transpose of each matrix
    Acm = A.transpose(1, 2).contiguous()
    w = torch.empty((B, n), dtype=torch.complex128, device=A.device)
    V = torch.empty((B, n, n), dtype=torch.complex128, device=A.device)
    info = (ctypes.c_int * B)()
    check(ctx.lib.sc_eigensolve_batched(ctx.handle, _ptr(Acm), n, B, _ptr(w), _ptr(V), info,
                                        _stream_ptr(stream)))
    return w, V.transpose(1, 2)      # V[b][:, j] is eigenvector j
