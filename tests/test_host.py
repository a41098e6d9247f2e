"""CPU checks of the host side: the C ABI library, the host plan, sharding.

None of these touch a GPU: the library is loaded and its symbols checked, and
sc_volume_plan (pure host arithmetic) is compared with the oracle's setup.
"""
import ctypes
import math
import os
import re
import subprocess

import numpy as np
import pytest

from oracle import scattervolume as osv
from scattersim_b200 import _lib, sweep

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "scattersim_b200.h")


@pytest.fixture(scope="module")
def lib():
    if not os.path.exists(_lib.LIB_PATH):
        subprocess.run(["make", "-C", os.path.join(ROOT, "scattersim_b200", "csrc"), "-j8"], check=True)
    return _lib.load()


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sc_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_function(lib):
    names = header_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), f"{name} declared in the header but not exported"
    # and the Python binding covers every declaration
    assert set(names) <= set(_lib.exported_symbols()), set(names) - set(_lib.exported_symbols())


def test_version_and_error_string(lib):
    assert lib.sc_version().startswith(b"scattersim_b200")
    assert isinstance(lib.sc_last_error_string(), bytes)


def test_params_defaults_match_reference_cli(lib):
    p = _lib.VolumeParams()
    lib.sc_volume_params_default(ctypes.byref(p))
    assert p.lambda_ == 1.0 and list(p.direction) == [0, 0, 1]
    assert list(p.ex) == [0, 0] and list(p.ey) == [1, 0] and list(p.ez) == [0, 0]
    assert list(p.n) == [1, 1] and p.kappa == 0.0 and list(p.size) == [10, 10, 2] and p.z == 0.0
    assert p.ncoef == 0 and p.psf == 0 and p.external == 0 and p.npz == 0


CASES = [
    dict(lambda_=0.5, size=(10, 10, 1), coef=(11, 11), ex=(1, 0), ey=(0, 0)),
    dict(lambda_=0.6, size=(20, 20, 8), coef=(21, 21),
         direction=(math.sin(math.radians(10)), 0, math.cos(math.radians(10))), ex=(1, 0), ey=(0, 0)),
    dict(lambda_=0.6, size=(5, 5, 1), coef=(21, 21)),           # evanescent clamp fires
    dict(lambda_=0.1, size=(10, 10, 1), coef=(31, 31)),          # pixel clamp
    dict(lambda_=0.7, size=(10, 10, 1), coef=(49,), direction=(0.2, -0.1, 1), ex=(0.3, 0.1), ey=(1, -0.2)),
    dict(lambda_=1.0, size=(10, 10, 10), coef=(1, 1), n=(1.0, 1.2), kappa=0.05),
]


@pytest.mark.parametrize("kw", CASES)
def test_plan_matches_oracle_setup(lib, kw):
    from scattersim_b200.solver import make_params, plan
    shape = (3, 20, 16) if kw.get("coef") == (31, 31) else (2, 64, 64)
    smp = np.ones(shape, dtype=complex)
    okw = dict(kw)
    if "kappa" in okw:
        okw["kappa"] = (okw["kappa"],)
    d, e, dirv, k, ni, slices, num_pixels, z, M, msgs = osv.setup(smp, osv.Params(**okw))
    dims = plan(make_params(**kw), shape)
    assert [dims.Mx, dims.My] == M
    assert dims.MF == M[0] * M[1]
    assert bool(dims.clamped) == bool(msgs)
    assert dims.k == k
    assert np.allclose(list(dims.dir), dirv, rtol=0, atol=1e-15)
    assert np.allclose(np.array(dims.e_re) + 1j * np.array(dims.e_im), e, rtol=0, atol=1e-15)


def test_plan_rejects_bad_input(lib):
    from scattersim_b200._lib import SC_BADINPUT
    from scattersim_b200.solver import make_params
    d = _lib.VolumeDims()
    p = make_params(lambda_=-1.0)
    assert lib.sc_volume_plan(ctypes.byref(p), 1, 8, 8, ctypes.byref(d)) == SC_BADINPUT
    p = make_params()
    assert lib.sc_volume_plan(ctypes.byref(p), 0, 8, 8, ctypes.byref(d)) == SC_BADINPUT
    p = make_params(direction=(0, 0, 0))
    assert lib.sc_volume_plan(ctypes.byref(p), 1, 8, 8, ctypes.byref(d)) == SC_BADINPUT


def test_lpt_assignment_is_a_partition_and_balanced():
    rng = np.random.default_rng(3)
    costs = [sweep.solve_cost(int(rng.integers(4, 17)), int(rng.choice([7, 11, 15, 21, 25])) ** 2)
             for _ in range(256)]
    for world in (1, 2, 3, 8):
        parts = sweep.assign_lpt(costs, world)
        flat = sorted(i for p in parts for i in p)
        assert flat == list(range(len(costs)))
        loads = [sum(costs[i] for i in p) for p in parts]
        assert max(loads) <= sum(costs) / world + max(costs)


def _gloo_worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    costs = [float(c) for c in (5, 1, 9, 3, 3, 7, 2, 8)]
    mine = sweep.shard(costs, rank, world)
    t = sweep.max_over_ranks(float(rank + 1), dist)
    import torch
    counts = torch.tensor([len(mine)], dtype=torch.int64)
    dist.all_reduce(counts)
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    q.put((rank, t, int(counts.item()), gathered))
    dist.destroy_process_group()


def test_two_rank_sharding_with_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_gloo_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for rank, t, count, gathered in res:
        assert t == 2.0                      # max over ranks of (rank + 1)
        assert count == 8                    # every instance solved exactly once
        flat = sorted(i for part in gathered for i in part)
        assert flat == list(range(8))


def test_wrapper_tensor_checks_run_before_the_library():
    """The solver wrappers refuse CPU tensors, wrong dtypes and wrong shapes before any pointer reaches the
    library (which reads as many elements as the sizes imply); checked on the CPU with a stand-in context."""
    import pytest
    import torch
    from scattersim_b200 import solver

    class Ctx:
        device = 0
    t = torch.zeros((2, 3), dtype=torch.complex128)
    with pytest.raises(TypeError, match="CUDA"):
        solver._checked(Ctx(), t, (2, 3), "E0")
    with pytest.raises(TypeError, match="complex128"):
        solver._checked(Ctx(), t.real, (2, 3), "E0")
    with pytest.raises(TypeError):
        solver.eigensolve(Ctx(), torch.zeros((2, 4, 4), dtype=torch.complex128))
    with pytest.raises(ValueError, match="square"):
        solver.eigensolve(Ctx(), torch.zeros((2, 4, 5), dtype=torch.complex128))
    with pytest.raises(ValueError, match="region bounds"):
        solver.evaluate(Ctx(), t, t, [0.0, 1.0], [0], [0], torch.zeros((4, 3)))
    with pytest.raises(TypeError):
        solver.sweep(Ctx(), [None], [torch.zeros((4, 4), dtype=torch.complex128)])


# entry points whose first statement refuses a null handle or buffer (no CUDA call comes before it)
NULL_CHECKED = [
    "sc_create", "sc_fft2_crop", "sc_phi", "sc_eigensolve_batched", "sc_linearsolve_batched", "sc_inverse_batched",
    "sc_zgemm_emulated_batched", "sc_zgemm_crt_batched", "sc_zgemm_batched", "sc_volume_plan", "sc_volume_solve",
    "sc_volume_chain_block", "sc_volume_boundary_solve", "sc_sweep_solve", "sc_kernel_timing", "sc_kernel_stats",
    "sc_kernel_stats_ex", "sc_gemm_choices_get", "sc_volume_precision", "sc_volume_stage_ms",
    "sc_fp64_peak_probe", "sc_fp64_dmma_probe", "sc_crt_tiles_set", "sc_int8_peak_probe", "sc_qr_stats",
    "sc_volume_waves", "sc_volume_field_grid", "sc_cw_write", "sc_cw_evaluate", "sc_beam_polar", "sc_layer_solve",
    "sc_mkl_eigensolve", "sc_gpu_initialize", "sc_linearsolve_batched_noalloc", "sc_scatterio_write",
    "sc_scatterio_read", "sc_fno_create", "sc_fno_status", "sc_fno_param_count", "sc_fno_params",
    "sc_fno_forward", "sc_fno_loss_grad", "sc_fno_train_step",
]


def test_null_arguments_are_refused_with_a_message(lib):
    """Every entry point above, called with null pointers and zero sizes, returns SC_BADINPUT and leaves a
    message for sc_last_error_string -- never a crash or an exit (the reference's HANDLE_ERROR exits)."""
    import ctypes
    for name in NULL_CHECKED:
        restype, argtypes = _lib._SIGS[name]
        args = []
        for t in argtypes:
            if t in (ctypes.c_double, ctypes.c_float):
                args.append(0.0)
            elif t in (ctypes.c_void_p, ctypes.c_char_p) or (isinstance(t, type) and issubclass(t, ctypes._Pointer)):
                args.append(None)
            else:
                args.append(0)
        rc = getattr(lib, name)(*args)
        assert rc == _lib.SC_BADINPUT, (name, rc)
        assert lib.sc_last_error_string(), name
