"""scattersim_b200: B200-native coupled-wave (RCWA) layer solve and field evaluation.

Drop-in for the scattervolume hot path of STIM-Lab/scattersim: Fourier
coefficients of each index slice, the 4M x 4M layer matrix, its
non-Hermitian eigendecomposition, the boundary / transfer-matrix solve and
the plane-wave field sum, all as hand-written sm_100a kernels behind the C ABI
of ``include/scattersim_b200.h``.

Python modules:
  ``solver``   -- ScatterVolume: the scattervolume options and solve
  ``cwfile``   -- CoupledWaveStructure and the .cw file format
  ``samples``  -- seeded synthetic samples of the benchmark workloads
"""
from ._lib import ScatterError, load  # noqa: F401

__all__ = ["ScatterError", "load"]
