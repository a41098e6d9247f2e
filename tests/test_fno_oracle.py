"""The surrogate's CPU oracle: its backward pass against finite differences.

Run in float64 (no BF16 rounding) so that central differences resolve the
gradient; the GPU network's gradients are then checked against this oracle in
its BF16 mode (tests/test_gpu_fno.py).
"""
import numpy as np

from oracle import fno as ofno


def random_params(seed=0, spectral_scale=2e-3):
    rng = np.random.default_rng(seed)
    lay = ofno.Layout()
    w = rng.uniform(-0.3, 0.3, lay.total)
    for l in range(ofno.L):
        n = ofno.NM * ofno.W * ofno.W
        w[lay.SWr[l]:lay.SWr[l] + n] = rng.uniform(0, spectral_scale, n)
        w[lay.SWi[l]:lay.SWi[l] + n] = rng.uniform(0, spectral_scale, n)
    return w, lay


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, -2.5e-3, 3.0e38], np.float32)
    r = ofno.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0   # tie to even
    assert r[2] == np.float32(1.0078125)
    assert abs(r[3] - x[3]) <= abs(x[3]) * 2 ** -8


def test_backward_matches_finite_differences():
    w, lay = random_params()
    rng = np.random.default_rng(1)
    maps = rng.uniform(1.0, 1.6, (2, 64, 64))
    lam = np.array([0.45, 0.7])
    tgt = rng.standard_normal((2, ofno.NOUT))
    net = ofno.Net(w, bf16_ops=False)
    _, g = net.loss_grad(maps, lam, tgt)
    picks = [lay.P + 3, lay.bP + 5, lay.Wl[1] + 77, lay.bl[3] + 2, lay.SWr[0] + 12345, lay.SWi[2] + 999,
             lay.SWr[3] + 4096 * 7 + 65, lay.Q1 + 300, lay.bQ1 + 9, lay.Q2 + 40, lay.bQ2 + 11]
    for idx in picks:
        h = 1e-5 * max(1.0, abs(w[idx]))
        wp, wm = w.copy(), w.copy()
        wp[idx] += h
        wm[idx] -= h
        lp = ofno.Net(wp, bf16_ops=False).loss_grad(maps, lam, tgt)[0].mean()
        lm = ofno.Net(wm, bf16_ops=False).loss_grad(maps, lam, tgt)[0].mean()
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[idx]) <= 1e-5 * max(1.0, abs(fd)) + 1e-7, (idx, fd, g[idx])
