"""ctypes binding of libscattersim_b200.so (the C ABI in include/scattersim_b200.h).

The library is built in-tree (``python -m scattersim_b200.build`` or
``__graft_entry__.build()``).  Loading fails loudly when it is missing: there
is no CPU fallback anywhere in the package.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_double, c_int, c_longlong, c_uint64, c_void_p, c_char_p

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libscattersim_b200.so")

SC_OK, SC_BADINPUT, SC_NOCONVERGE, SC_SINGULAR, SC_OOM, SC_CUDA_ERROR, SC_ENERGY_FAIL = range(7)
STATUS_NAMES = {0: "SC_OK", 1: "SC_BADINPUT", 2: "SC_NOCONVERGE", 3: "SC_SINGULAR", 4: "SC_OOM",
                5: "SC_CUDA_ERROR", 6: "SC_ENERGY_FAIL"}


SC_SWEEP_FP64 = 0
SC_SWEEP_MIXED = 1
SC_SWEEP_CRT = 2


def SC_SWEEP_SLICES(s):
    return 0x100 | int(s)


class ScatterError(RuntimeError):
    """A C-ABI call returned a non-OK sc_status."""

    def __init__(self, status, msg):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {msg}")
        self.status = status


class VolumeParams(ctypes.Structure):
    """sc_volume_params (the scattervolume options, ScatterVolume.cpp:511-529)."""
    _fields_ = [("lambda_", c_double), ("direction", c_double * 3), ("ex", c_double * 2),
                ("ey", c_double * 2), ("ez", c_double * 2), ("n", c_double * 2), ("kappa", c_double),
                ("size", c_double * 3), ("z", c_double), ("ncoef", c_int), ("coef", c_int * 2),
                ("psf", c_int), ("external", c_int), ("npz", c_int)]


class VolumeDims(ctypes.Structure):
    """sc_volume_dims."""
    _fields_ = [("Mx", c_int), ("My", c_int), ("MF", c_int), ("Z", c_int), ("clamped", c_int),
                ("k", c_double), ("dir", c_double * 3), ("e_re", c_double * 3), ("e_im", c_double * 3)]


# name -> (restype, argtypes)
_SIGS = {
    "sc_version": (c_char_p, []),
    "sc_last_error_string": (c_char_p, []),
    "sc_create": (c_int, [POINTER(c_void_p), c_int]),
    "sc_destroy": (c_int, [c_void_p]),
    "sc_launch_count": (c_uint64, [c_void_p]),
    "sc_fft2_crop": (c_int, [c_void_p, c_void_p, c_int, c_int, c_int, c_int, c_int, c_void_p, c_void_p, c_void_p]),
    "sc_phi": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_int, c_int, POINTER(c_double), POINTER(c_double),
                       c_double, c_void_p, c_void_p]),
    "sc_eigensolve_batched": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p, POINTER(c_int),
                                      c_void_p]),
    "sc_linearsolve_batched": (c_int, [c_void_p, c_void_p, c_int, c_void_p, c_int, c_int, POINTER(c_int),
                                       c_void_p]),
    "sc_linearsolve_batched_noalloc": (c_int, [c_void_p, c_int, c_void_p, c_int, c_int, POINTER(c_int),
                                               c_void_p]),
    "sc_inverse_batched": (c_int, [c_void_p, c_void_p, c_int, c_int, c_void_p, POINTER(c_int), c_void_p]),
    "sc_zgemm_emulated_batched": (c_int, [c_void_p, c_int, c_int, c_int, c_int, POINTER(c_double), c_void_p, c_int, c_longlong,
                                 c_void_p, c_int, c_longlong, POINTER(c_double), c_void_p, c_int, c_longlong,
                                 c_int, c_void_p]),
    "sc_zgemm_crt_batched": (c_int, [c_void_p, c_int, c_int, c_int, POINTER(c_double), c_void_p, c_int, c_longlong,
                                     c_void_p, c_int, c_longlong, POINTER(c_double), c_void_p, c_int, c_longlong,
                                     c_int, c_void_p]),
    "sc_zgemm_batched": (c_int, [c_void_p, c_int, c_int, c_int, POINTER(c_double), c_void_p, c_int, c_longlong,
                                 c_void_p, c_int, c_longlong, POINTER(c_double), c_void_p, c_int, c_longlong,
                                 c_int, c_void_p]),
    "sc_scatterio_write": (c_int, [ctypes.c_char_p, POINTER(c_double), POINTER(c_double), c_int, POINTER(c_longlong),
                                   c_void_p, c_void_p, c_void_p]),
    "sc_scatterio_read": (c_int, [ctypes.c_char_p, POINTER(c_double), POINTER(c_double), POINTER(c_int),
                                  POINTER(c_longlong), c_int, c_void_p, c_void_p, c_void_p, c_longlong,
                                  POINTER(c_longlong)]),
    "sc_volume_chain_block": (c_int, [c_void_p, POINTER(VolumeParams), c_void_p, c_int, c_int, c_int, c_int, c_int,
                                      c_void_p, c_void_p, POINTER(c_int), c_void_p]),
    "sc_volume_boundary_solve": (c_int, [c_void_p, POINTER(VolumeParams), c_int, c_int, c_int, c_void_p, c_void_p,
                                         c_void_p, POINTER(c_int), c_void_p]),
    "sc_volume_field_grid": (c_int, [c_void_p, POINTER(VolumeParams), c_int, c_int, c_int, c_void_p, c_void_p,
                                     c_void_p, c_void_p, c_int, POINTER(c_double), POINTER(c_double), POINTER(c_int),
                                     c_double, c_void_p, c_int, c_void_p]),
    "sc_cw_write": (c_int, [c_void_p, ctypes.c_char_p, c_void_p, c_void_p, c_longlong, c_int, POINTER(c_double),
                            POINTER(c_longlong), c_int, c_void_p]),
    "sc_volume_params_default": (None, [POINTER(VolumeParams)]),
    "sc_volume_plan": (c_int, [POINTER(VolumeParams), c_int, c_int, c_int, POINTER(VolumeDims)]),
    "sc_sweep_solve": (c_int, [c_void_p, c_int, POINTER(VolumeParams), POINTER(c_void_p), POINTER(c_int),
                               POINTER(c_int), POINTER(c_int), POINTER(c_void_p), c_int, POINTER(c_int), c_void_p]),
    "sc_kernel_timing": (c_int, [c_void_p, c_int]),
    "sc_kernel_stats": (c_int, [c_void_p, POINTER(c_double)]),
    "sc_kernel_stats_ex": (c_int, [c_void_p, POINTER(c_double), c_int]),
    "sc_gemm_choices_get": (c_int, [c_void_p, POINTER(c_int), c_int, POINTER(c_int)]),
    "sc_gemm_choices_set": (c_int, [c_void_p, POINTER(c_int), c_int]),
    "sc_fno_create": (c_int, [POINTER(c_void_p), c_int, c_int, ctypes.c_ulonglong]),
    "sc_fno_destroy": (c_int, [c_void_p]),
    "sc_fno_param_count": (c_int, [c_void_p, POINTER(c_longlong)]),
    "sc_fno_status": (c_int, [c_void_p]),
    "sc_fno_params": (c_int, [c_void_p, c_void_p, c_int, c_void_p]),
    "sc_fno_forward": (c_int, [c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p]),
    "sc_fno_loss_grad": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_void_p]),
    "sc_fno_train_step": (c_int, [c_void_p, c_void_p, c_void_p, c_void_p, c_int, ctypes.c_float, c_void_p,
                                  c_void_p]),
    "sc_volume_precision": (c_int, [c_void_p, c_int]),
    "sc_volume_solve": (c_int, [c_void_p, POINTER(VolumeParams), c_void_p, c_int, c_int, c_int, c_void_p,
                                c_void_p, c_void_p, c_void_p, POINTER(c_int), c_void_p]),
    "sc_volume_stage_ms": (c_int, [c_void_p, POINTER(c_double)]),
    "sc_fp64_peak_probe": (c_int, [c_void_p, POINTER(c_double)]),
    "sc_fp64_dmma_probe": (c_int, [c_void_p, POINTER(c_double)]),
    "sc_int8_peak_probe": (c_int, [c_void_p, POINTER(c_double)]),
    "sc_crt_tiles_set": (c_int, [c_void_p, c_int]),
    "sc_qr_stats": (c_int, [c_void_p, POINTER(c_longlong), c_int]),
    "sc_volume_waves": (c_int, [c_void_p, POINTER(VolumeParams), c_int, c_int, c_int, c_void_p, c_void_p,
                                c_void_p, c_void_p, c_int, POINTER(c_longlong), POINTER(c_int), POINTER(c_int),
                                POINTER(c_double), c_void_p, c_void_p, c_void_p]),
    "sc_cw_evaluate": (c_int, [c_void_p, c_void_p, c_void_p, c_int, POINTER(c_double), POINTER(c_int),
                               POINTER(c_int), c_int, c_double, c_void_p, c_longlong, c_void_p, c_int, c_void_p]),
    "sc_mkl_eigensolve": (c_int, [c_void_p, c_void_p, c_void_p, c_int]),
    "sc_beam_polar": (c_int, [c_void_p, c_double, c_double, c_int, c_int, POINTER(c_double), POINTER(c_double),
                              POINTER(c_double), c_void_p, c_void_p, POINTER(c_int), c_void_p]),
    "sc_layer_solve": (c_int, [c_void_p, c_int, POINTER(c_double), POINTER(c_double), POINTER(c_double), c_double,
                               c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                               c_void_p]),
    "sc_gpu_initialize": (c_int, [c_int, POINTER(ctypes.c_float), POINTER(c_int), POINTER(c_int), c_void_p,
                                  c_longlong, c_int]),
    "sc_gpu_cw_evaluate": (c_int, [c_void_p, c_void_p, c_void_p, ctypes.c_float, ctypes.c_float, ctypes.c_float,
                                   ctypes.c_float, ctypes.c_float, ctypes.c_float, ctypes.c_float, c_int, c_int]),
}

_lib = None


def load():
    """Load the shared library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m scattersim_b200.build` "
                          "(the package has no CPU fallback)")
    lib = ctypes.CDLL(LIB_PATH)
    for name, (res, args) in _SIGS.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def exported_symbols():
    """Names the header declares (for the export test)."""
    return list(_SIGS.keys())


def check(status):
    if status != SC_OK:
        msg = load().sc_last_error_string().decode(errors="replace")
        raise ScatterError(status, msg)
    return status
