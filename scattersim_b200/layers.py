"""scatterlayer / scatterplane: homogeneous-layer solves of a focused beam through the C ABI.

Mirrors the two reference programs' option surfaces and main() flows with the
same names and defaults:

* ``scatterlayer`` -- ScatterLayer.cpp:281-420: --lambda --direction --ex --ey
  --ez --n --kappa --z --alpha --beta --na --samples (polar mode);
* ``scatterplane`` -- ScatterPlane.cpp:81-264: --lambda --direction --focus
  --ex --ey --ez --n --kappa --z --alpha --beta --samples --wavemask (polar
  mode), the one-interface (L = 2) case of the same solve.

The beam (``sc_beam_polar``) and every per-wave system (``sc_layer_solve``)
run on the GPU; this module only pads the option lists and orthogonalises the
polarisation as the reference's main() does.  Results are device tensors with
Cartesian E0; ``cwfile`` stores them in the record frame of the reference's
.cw files.
"""
from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np
import torch

from ._lib import check
from .solver import Context, _ptr, _stream_ptr

LAYER_MAX = 15


def fill_layers(n, kappa, z):
    """ScatterLayer.cpp:328-343: L = the longest of n, kappa + 1, z + 1; pad the other lists."""
    n, kappa, z = [float(v) for v in n], [float(v) for v in kappa], [float(v) for v in z]
    L = max(len(n), len(kappa) + 1, len(z) + 1)
    n += [n[-1]] * (L - len(n))
    kappa = (kappa + [0.0] * L)[:L - 1]
    while len(z) + 1 < L:
        z.append(z[-1] + 10.0)
    return L, n, kappa, z[:L - 1]


def orthogonalize(e, d):
    """FourierWave.h:32-39, applied by both programs (ScatterLayer.cpp:349, ScatterPlane.cpp:132):
    E /= sqrt(Ex^2 + Ey^2 + Ez^2) (complex squares, no conjugate), then d x (E x d)."""
    e = np.asarray(e, dtype=np.complex128)
    e = e / np.sqrt(e[0] ** 2 + e[1] ** 2 + e[2] ** 2)
    d = np.asarray(d, dtype=np.complex128)
    return np.cross(d, np.cross(e, d))


def _centre(lambda_, direction, ex, ey, ez, n0):
    """Centre wave: k = dir n0 2 pi / lambda (ScatterLayer.cpp:345-353; ScatterPlane.cpp:134 forms
    k = 2 pi n0 / lambda with the unit direction, the same vector), E orthogonalised."""
    d = np.asarray(direction, dtype=np.float64)
    d = d / np.linalg.norm(d)
    e = orthogonalize(np.array([complex(*ex), complex(*ey), complex(*ez)]), d)
    return d * n0 * (2 * math.pi / lambda_), e


@dataclass
class BeamSolution:
    Pi_k: torch.Tensor       # (N, 3) float64 incident wave vectors
    Pi_E: torch.Tensor       # (N, 3) complex128 incident E0 (wound to the focal point)
    z: list                  # boundary planes
    Pr_E: torch.Tensor       # (N, L-1, 3) complex128, reflected E0 per boundary (wound by -z_l)
    Pr_k: torch.Tensor
    Pt_E: torch.Tensor       # (N, L-1, 3) complex128, transmitted E0 per boundary (wound by -z_l)
    Pt_k: torch.Tensor


def beam(ctx: Context, lambda_, k_center, e_center, alpha, beta, samples, focus=(0.0, 0.0, 0.0), stream=None):
    """The focused beam of SolidAnglePolar on the device: (k (N, 3) float64, E0 (N, 3) complex128)."""
    N0, N1 = _samples(samples)
    dev = torch.device("cuda", ctx.device)
    kout = torch.empty((N0 * N1, 3), dtype=torch.float64, device=dev)
    Eout = torch.empty((N0 * N1, 3), dtype=torch.complex128, device=dev)
    kc = (ctypes.c_double * 3)(*[float(v) for v in k_center])
    ec = np.asarray(e_center, dtype=np.complex128)
    ecb = (ctypes.c_double * 6)(*[v for c in ec for v in (c.real, c.imag)])
    fc = (ctypes.c_double * 3)(*[float(v) for v in focus])
    cnt = ctypes.c_int(0)
    check(ctx.lib.sc_beam_polar(ctx.handle, float(alpha), float(beta), N0, N1, kc, ecb, fc, _ptr(kout), _ptr(Eout),
                                ctypes.byref(cnt), _stream_ptr(stream)))
    return kout[:cnt.value], Eout[:cnt.value]


def _samples(samples):
    """ScatterLayer.cpp:355-376: one value = a square grid (polar mode)."""
    if len(samples) == 1:
        s = int(math.sqrt(samples[0]))
        return s, s
    return int(samples[0]), int(samples[1])


def layer_solve(ctx: Context, k_in: torch.Tensor, E_in: torch.Tensor, n, kappa, z, lambda_, stream=None):
    """sc_layer_solve over (N, 3) incident waves: per boundary reflected / transmitted (E0, k)."""
    L = len(n)
    N = int(k_in.shape[0])
    dev = k_in.device
    nb = max(L - 1, 0)
    out = [torch.empty((N, nb, 3), dtype=torch.complex128, device=dev) for _ in range(4)]
    na = (ctypes.c_double * L)(*n)
    ka = (ctypes.c_double * max(L - 1, 1))(*(list(kappa) or [0.0]))
    za = (ctypes.c_double * max(L - 1, 1))(*(list(z) or [0.0]))
    status = torch.zeros(max(N, 1), dtype=torch.int32, device=dev)
    check(ctx.lib.sc_layer_solve(ctx.handle, L, na, ka, za, float(lambda_), N, _ptr(k_in.contiguous()),
                                 _ptr(E_in.contiguous()), _ptr(out[0]), _ptr(out[1]), _ptr(out[2]), _ptr(out[3]),
                                 _ptr(status), _stream_ptr(stream)))
    return out


def scatterlayer(ctx: Context, lambda_=1.0, direction=(0, 0, 1), ex=(0, 0), ey=(1, 0), ez=(0, 0),
                 n=(1, 1.4, 1.4, 1.0), kappa=(0.05,), z=(-5.0, 0.0, 5.0), alpha=1.0, beta=0.0, na=None,
                 samples=(64, 64), stream=None) -> BeamSolution:
    """ScatterLayer.cpp:281-420 (polar mode) on the GPU."""
    L, n, kappa, z = fill_layers(n, kappa, z)
    if L > LAYER_MAX:
        raise ValueError(f"at most {LAYER_MAX} layers")
    if na is not None:
        alpha = math.asin(na / n[0])                                         # :324-326
    kc, e = _centre(lambda_, direction, ex, ey, ez, n[0])
    ks, Es = beam(ctx, lambda_, kc, e, alpha, beta, samples, stream=stream)
    rE, rk, tE, tk = layer_solve(ctx, ks, Es, n, kappa, z, lambda_, stream)
    return BeamSolution(ks, Es, z, rE, rk, tE, tk)


def scatterplane(ctx: Context, lambda_=1.0, direction=(1, 0, 1), focus=(0, 0, 0), ex=(0, 0), ey=(1, 0), ez=(0, 0),
                 n=(1.0, 1.4), kappa=0.05, z=0.0, alpha=0.5, beta=0.0, samples=(64, 64),
                 stream=None) -> BeamSolution:
    """ScatterPlane.cpp:81-264 (polar mode) on the GPU: the L = 2 layer solve at plane z."""
    kc, e = _centre(lambda_, direction, ex, ey, ez, n[0])
    ks, Es = beam(ctx, lambda_, kc, e, alpha, beta, samples, focus=focus, stream=stream)
    rE, rk, tE, tk = layer_solve(ctx, ks, Es, [float(n[0]), float(n[1])], [float(kappa)], [float(z)], lambda_,
                                 stream)
    return BeamSolution(ks, Es, [float(z)], rE, rk, tE, tk)
