"""Host-side logic of the surrogate, on the CPU: sample generation, target
packing and the energy-balance check (pinned by oracle solves)."""
import numpy as np

from oracle import scattervolume as osv
from scattersim_b200 import surrogate as sg


def test_instances_are_seeded_and_in_range():
    a, la = sg.instance(7)
    b, lb = sg.instance(7)
    c, _ = sg.instance(8)
    assert np.array_equal(a, b) and la == lb and not np.array_equal(a, c)
    assert a.shape == (64, 64) and 1.0 <= a.min() and a.max() <= 1.6 and 0.4 <= la <= 0.8


def test_target_packing_roundtrip():
    rng = np.random.default_rng(0)
    x = rng.standard_normal(726) + 1j * rng.standard_normal(726)
    t = sg.x_to_target(x)
    assert t.shape == (sg.NOUT,) and t.dtype == np.float32
    assert np.allclose(sg.target_to_x(t)[0], x, atol=1e-6)


def test_energy_error_of_oracle_solves_is_zero():
    """Lossless maps at normal incidence, x-pol: sum |R|^2 Sz + |T|^2 Sz = 1 for the oracle's x."""
    xs, lams = [], []
    for seed in (3, 4):
        m, lam = sg.instance(seed)
        p = osv.Params(lambda_=lam, size=(sg.PERIOD, sg.PERIOD, sg.SLAB), coef=(sg.ORDERS, sg.ORDERS),
                       ex=(1.0, 0.0), ey=(0.0, 0.0), external=True)
        xs.append(osv.solve(m.reshape(1, 64, 64).astype(complex), p, keep=False).x)
        lams.append(lam)
    err = sg.energy_error(np.stack(xs), np.array(lams))
    assert err.max() < 1e-9
    # and it detects a 1 % amplitude error
    assert (sg.energy_error(np.stack(xs) * 1.01, np.array(lams)) > 1e-3).all()


def test_network_buffers_are_checked_before_the_library():
    """The library reads batch x 64 x 64 maps, batch wavelengths and batch x 1452 targets from bare pointers:
    the wrapper converts and places them on the network's device, and refuses a wrong shape."""
    import pytest
    import torch
    net = sg.Surrogate.__new__(sg.Surrogate)        # no library handle: only the buffer checks run
    net.device = torch.device("cpu")
    maps = np.ones((3, 64, 64))
    B, (m, lam, t) = net._batch(maps, [0.5, 0.6, 0.7], np.zeros((3, sg.NOUT)))
    assert B == 3 and m.dtype == lam.dtype == t.dtype == torch.float32
    assert m.is_contiguous() and tuple(m.shape) == (3, 64, 64) and tuple(t.shape) == (3, sg.NOUT)
    with pytest.raises(ValueError, match="maps"):
        net._batch(np.ones((3, 32, 32)), [0.5, 0.6, 0.7])
    with pytest.raises(ValueError, match="lams"):
        net._batch(maps, [0.5, 0.6])
    with pytest.raises(ValueError, match="target"):
        net._batch(maps, [0.5, 0.6, 0.7], np.zeros((3, sg.NOUT - 2)))
    with pytest.raises(ValueError, match="no network"):
        sg.predict_with_fallback([], None, maps, [0.5, 0.6, 0.7])
