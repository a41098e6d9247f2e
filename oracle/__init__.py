"""CPU oracle for the scattervolume hot path (test infrastructure only).

This package is a numpy/scipy restatement of the reference's CPU algorithm
(ScatterVolume.cpp, FourierWave.h, third_Lapack.h, CoupledWaveStructure.h,
ScatterIO.h, cpuEvaluator.cpp, gpuEvaluator.cu).  It is the checker for the CUDA path and
the timed CPU baseline; nothing in the product package imports it.

Parity pin status
-----------------
* ``.cw`` byte layout: pinned by the reference's own output files
  ``data/psf.cw`` and ``x64/a.cw`` (parse/round-trip to the last byte).
* scattervolume numerics at M = 1: pinned by the closed-form multilayer
  Fresnel restatement of ``ScatterLayer.cpp:152-232`` (the consistency the
  reference states in ``data/generate_layer_volume.py:1-2``).
* scattervolume numerics at M > 1: the reference ships no output, so the
  restatement itself (LAPACK zgeev/zgesv through scipy standing in for MKL)
  plus physics invariants (energy balance, field continuity) is the pin.
  Parity at M > 1 is therefore "pinned to the restatement, not to a reference
  run" -- the reference cannot be built here (Eigen, MKL, FFTW, Boost, tira
  are absent).
"""
