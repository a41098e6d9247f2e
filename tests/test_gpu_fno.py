"""The surrogate network on the GPU against its CPU oracle, and its fallback.

Forward outputs and every parameter group's gradient are compared with
oracle/fno.py in its BF16 mode (operands rounded to BF16 at the same points,
FP32 storage); the GPU accumulates in FP32 and the oracle in FP64, so a few
BF16 roundings of intermediate values can differ -- the bounds are relative
norms per group.  Training must lower the loss, and the fallback must return
the plain solve's answer wherever the energy check fails.
"""
import numpy as np
import pytest
import torch

from oracle import fno as ofno
from scattersim_b200 import surrogate as sg

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def net():
    s = sg.Surrogate(0, max_batch=64, seed=3)
    yield s
    s.close()


def random_params(seed=0):
    rng = np.random.default_rng(seed)
    lay = ofno.Layout()
    w = rng.uniform(-0.3, 0.3, lay.total).astype(np.float32)
    for l in range(ofno.L):
        n = ofno.NM * ofno.W * ofno.W
        w[lay.SWr[l]:lay.SWr[l] + n] = rng.uniform(0, 2e-3, n)
        w[lay.SWi[l]:lay.SWi[l] + n] = rng.uniform(0, 2e-3, n)
    return w, lay


def batch(seed=1, B=2):
    rng = np.random.default_rng(seed)
    maps = np.stack([sg.surrogate_map(rng) for _ in range(B)]).astype(np.float32)
    lams = rng.uniform(0.4, 0.8, B).astype(np.float32)
    tgt = rng.standard_normal((B, ofno.NOUT)).astype(np.float32)
    return maps, lams, tgt


def test_forward_matches_oracle(net):
    w, _ = random_params()
    net.set_params(w)
    maps, lams, _ = batch()
    got = net.forward(torch.from_numpy(maps).cuda(), torch.from_numpy(lams).cuda()).cpu().numpy()
    net.status()
    ref = ofno.Net(w).forward(maps, lams)
    assert np.linalg.norm(got - ref) <= 5e-3 * np.linalg.norm(ref)


def test_gradients_match_oracle(net):
    w, lay = random_params(4)
    net.set_params(w)
    maps, lams, tgt = batch(5)
    loss, grad = net.loss_grad(torch.from_numpy(maps).cuda(), torch.from_numpy(lams).cuda(),
                               torch.from_numpy(tgt).cuda())
    net.status()
    rl, rg = ofno.Net(w).loss_grad(maps, lams, tgt)
    assert np.allclose(loss.cpu().numpy(), rl, rtol=5e-3)
    g = grad.cpu().numpy()
    groups = [("P", lay.P, ofno.W * ofno.CIN), ("bP", lay.bP, ofno.W), ("Q1", lay.Q1, ofno.HID * ofno.W),
              ("bQ1", lay.bQ1, ofno.HID), ("Q2", lay.Q2, ofno.COUT * ofno.HID), ("bQ2", lay.bQ2, ofno.COUT)]
    for l in range(ofno.L):
        groups += [(f"W{l}", lay.Wl[l], ofno.W * ofno.W), (f"b{l}", lay.bl[l], ofno.W),
                   (f"SWr{l}", lay.SWr[l], ofno.NM * ofno.W * ofno.W), (f"SWi{l}", lay.SWi[l], ofno.NM * ofno.W * ofno.W)]
    for name, off, n in groups:
        a, b = g[off:off + n], rg[off:off + n]
        assert np.linalg.norm(a - b) <= 2e-2 * np.linalg.norm(b) + 1e-12, (name, np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.fixture(scope="module")
def solved(ctx):
    maps, lams, xs = sg.generate(ctx, range(500, 532))
    return maps, lams, xs


def test_plain_targets_conserve_energy(solved):
    _, lams, xs = solved
    assert sg.energy_error(xs, lams).max() < 1e-9


def test_training_lowers_loss(net, solved):
    maps, lams, xs = solved
    tgt = np.stack([sg.x_to_target(x) for x in xs])
    fresh = sg.Surrogate(0, max_batch=32, seed=11)
    dm, dl, dt = (torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in (maps, lams, tgt))
    first = float(fresh.train_step(dm, dl, dt, 1e-3).mean())
    for _ in range(150):
        last = float(fresh.train_step(dm, dl, dt, 1e-3).mean())
    fresh.status()
    fresh.close()
    assert last < 0.2 * first, (first, last)


def test_fallback_returns_plain_solve(net, ctx, solved):
    """An untrained network fails the energy check everywhere; every answer is then the plain solve's."""
    maps, lams, xs = solved
    fresh = sg.Surrogate(0, max_batch=32, seed=12)
    out, bad = sg.predict_with_fallback(fresh, ctx, maps[:8], lams[:8])
    fresh.close()
    assert bad.all()
    assert np.max(sg.rel_err(out, xs[:8])) < 1e-12
