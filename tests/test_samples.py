"""The seeded synthetic workloads the bench and the parity tests solve (no GPU).

Shapes, dtypes and value ranges of each generator, determinism per seed, the
sweep's strata (wavelengths, angles, order counts, stack depths), and that the
reference's order clamp (ScatterVolume.cpp:612-651, restated in the oracle)
never changes the sweep's order counts, the premise of its 25 um period.
"""
import numpy as np
import pytest

from oracle import scattervolume as osv
from scattersim_b200 import samples


def test_triangle_map_is_seeded_and_binary():
    a, b, c = samples.triangle_map(3), samples.triangle_map(3), samples.triangle_map(4)
    assert a.shape == (1, 64, 64) and a.dtype == np.complex128
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    vals = set(np.unique(a).tolist())
    assert vals <= {1.0 + 0j, 1.4 + 0j} and len(vals) == 2
    # the triangle covers at least its minimum area of 5 um^2 of the 100 um^2 period, up to pixel sampling
    assert (a == 1.4).mean() * 100.0 > 4.0


def test_sphere_volume_ranges():
    v = samples.sphere_volume(7, nxy=48, nz=12)
    assert v.shape == (12, 48, 48) and v.dtype == np.complex128
    assert np.array_equal(v, samples.sphere_volume(7, nxy=48, nz=12))
    inside = v != 1.0
    assert inside.any()
    assert np.all((v.real[inside] >= 1.3) & (v.real[inside] <= 1.6))
    assert np.all((v.imag >= 0.0) & (v.imag <= 0.02))
    assert len(np.unique(v[inside])) <= 12


def test_disk_stack_ranges():
    for seed in range(20):
        maps, thick = samples.disk_stack(seed, n=32)
        assert 4 <= maps.shape[0] <= 16 and maps.shape[1:] == (32, 32)
        assert 0.1 <= thick <= 0.5
        assert np.all((maps.real >= 1.0) & (maps.real <= 1.6)) and np.all(maps.imag == 0)


def test_sweep_strata():
    inst = samples.sweep_instances(5, count=256, n=16)
    assert len(inst) == 256
    lams = [it.wavelength for it in inst]
    assert all(0.4 <= l <= 0.8 for l in lams)
    assert len(set(lams)) == 64 and lams[::4] == sorted(lams[::4])       # 64 sorted wavelengths
    assert [it.angle_deg for it in inst[:8]] == [0.0, 10.0, 20.0, 30.0] * 2
    assert {it.orders for it in inst} == set(samples.ORDER_CHOICES)
    assert all(it.period == 25.0 and it.params_kw()["external"] for it in inst)
    again = samples.sweep_instances(5, count=256, n=16)
    assert all(np.array_equal(a.maps, b.maps) and a.orders == b.orders for a, b in zip(inst, again))


@pytest.mark.parametrize("lam,angle", [(0.8, 30.0), (0.4, 30.0), (0.8, 0.0)])
def test_order_clamp_never_fires_on_the_sweep(lam, angle):
    """At the largest order count (25 x 25) over the 25 um period, the extreme wavelength and angle keep every
    order: the reference's clamp leaves M as requested."""
    it = samples.sweep_instances(1, count=4, n=64)[0]            # the workload's 64 x 64 maps (M <= pixels)
    it.wavelength, it.angle_deg, it.orders = lam, angle, 25
    *_, M, msgs = osv.setup(it.maps, osv.Params(**it.params_kw()))
    assert tuple(M) == (25, 25) and not msgs


def test_order_clamp_fires_below_the_sweep_period():
    """The control: at 23 um (below the 23.3 um the worst case needs) the clamp cuts the 25 x 25 orders."""
    it = samples.sweep_instances(1, count=4, n=64, period=23.0)[0]
    it.wavelength, it.angle_deg, it.orders = 0.8, 30.0, 25
    *_, M, msgs = osv.setup(it.maps, osv.Params(**it.params_kw()))
    assert tuple(M) != (25, 25) and msgs
