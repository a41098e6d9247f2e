"""Host-side logic of the scatterlayer / scatterplane mirror (no GPU): the layer-list
padding of ScatterLayer.cpp:328-343, the polarisation clean-up of FourierWave.h:32-39
and the centre wave, against the oracle's restatement."""
import numpy as np
import pytest

from oracle import scatterlayer as osl
from scattersim_b200 import layers


@pytest.mark.parametrize("n,kappa,z", [
    ((1, 1.4, 1.4, 1.0), (0.05,), (-5.0, 0.0, 5.0)),       # the reference's defaults
    ((1.0,), (0.1, 0.2), ()),                              # kappa decides L; z padded by 10
    ((1.0, 1.5), (), (-1.0, 0.0, 2.0, 3.0)),               # z decides L; n padded with its last value
    ((1.2,), (), ()),                                      # one layer
])
def test_fill_layers_matches_oracle(n, kappa, z):
    L, nn, kk, zz = layers.fill_layers(n, kappa, z if z else ([0.0] if len(kappa) else []))
    oL, on, ok, oz, ri = osl.fill_layers(n, kappa, z if z else ([0.0] if len(kappa) else []))
    assert (L, nn, kk, zz) == (oL, on, ok, oz)
    assert len(nn) == L and len(kk) == L - 1 and len(zz) == L - 1


@pytest.mark.parametrize("direction,ex,ey,ez,n0", [
    ((0, 0, 1), (0, 0), (1, 0), (0, 0), 1.0),
    ((1, 0, 1), (0.3, 0.1), (1, 0), (0, 0.2), 1.0),
    ((0.2, -0.4, 1), (1, 0), (0, 0), (0, 0), 1.33),
])
def test_centre_wave_matches_oracle(direction, ex, ey, ez, n0):
    k, e = layers._centre(0.7, direction, ex, ey, ez, n0)
    ok, oe = osl.incident(0.7, direction, ex, ey, ez, n0)
    assert np.allclose(k, ok, rtol=0, atol=1e-14) and np.allclose(e, oe, rtol=0, atol=1e-14)
    d = np.asarray(direction, float) / np.linalg.norm(direction)
    assert abs(np.dot(e, d)) < 1e-14                        # transverse after the clean-up


def test_samples_rule():
    assert layers._samples((64, 64)) == (64, 64)
    assert layers._samples((375,)) == (19, 19)              # one value: a square grid (polar mode)
