"""The learned Drucker-Prager projection: labels, the network's tensor-core
training and inference kernels against the NumPy oracle, and what training
gains over the untrained network."""
import numpy as np
import pytest

import icempm_b200 as im
from icempm_b200 import surrogate as sg
from oracle import mlp_oracle as mo
from oracle import oracle as orc

from mpm_cases import params


def _net(seed=0, x=None, y=None):
    net = sg.init_net(seed)
    if x is not None:
        v = sg.views(net)
        v["x_mu"][:] = x.mean(0)
        sd = x.std(0)
        v["x_sd"][:] = np.where(sd > 1e-6 * np.maximum(1, np.abs(x.mean(0))), sd, 1.0)
        v["y_mu"][:] = y.mean(0)
        v["y_sd"][:] = np.maximum(y.std(0), 1e-6)
    return net


@pytest.fixture(scope="module")
def pairs():
    p = params()
    x, y = mo.synthetic_pairs(p, 6000, seed=3)
    return p, x, y


def test_dp_project_matches_oracle_constitutive():
    """The principal-space restatement equals the full FP64 oracle on
    crushed particles with diagonal Fe (U = V = I), every branch."""
    p = params()
    m = mo.material(p)
    rng = np.random.default_rng(5)
    seen = set()
    for _ in range(400):
        a, b = 1.0 + rng.uniform(-5e-3, 5e-3, 2)
        s0, s1 = max(a, b), min(a, b)
        jp = rng.uniform(0.99, 1.02)
        ch, s0n, s1n, jpn = mo.dp_project(m["kappa"], m["mu"], m["p_thr"], m["tan_phi"], m["pmax"], m["qmax"], s0, s1,
                                          jp)
        Fe, jp2, cr, _, _ = orc.constitutive(p, np.array([s0, 0, 0, s1]), jp, 1, 0)
        seen.add((jp < 1 or s0 * s1 > 1.00001, ch))
        assert cr == 1
        assert abs(Fe[0] - s0n) <= 1e-12 and abs(Fe[3] - s1n) <= 1e-12 and abs(Fe[1]) <= 1e-12
        assert abs(jp2 - jpn) <= 1e-12
    assert len(seen) >= 3


def test_oracle_backward_matches_finite_differences(pairs):
    _, x, y = pairs
    x, y = x[:64], y[:64]
    net = _net(1, x, y)
    g, _ = mo.backward(net, x, y, exact=True)
    rng = np.random.default_rng(0)
    for i in rng.choice(sg.OFF_XMU, 40, replace=False):
        e = 1e-2
        a, b = net.copy(), net.copy()
        a[i] += e
        b[i] -= e
        fd = (mo.loss(a, x, y, exact=True) - mo.loss(b, x, y, exact=True)) / (2 * e)
        assert abs(fd - g[i]) <= 2e-3 * max(1.0, abs(g).max()), (i, fd, g[i])


def test_bf16_rounding():
    a = np.array([1.0, 1.00390625, 1.0 + 2 ** -8 + 2 ** -9, -3.14159], np.float32)
    r = mo._round(a)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == np.float32(1.0 + 2 ** -7)
    assert abs(r[3] + 3.140625) < 1e-6


@pytest.mark.gpu
def test_gradient_kernel_matches_oracle(pairs):
    """One forward/backward pass of the tcgen05 training kernel against the
    oracle with the same BF16 rounding (1000 samples: 8 tiles, the last
    partial)."""
    _, x, y = pairs
    x, y = x[:1000], y[:1000]
    net = _net(2, x, y)
    g_gpu, loss_gpu = sg.gradient(net, x, y)
    g_ref, loss_ref = mo.backward(net, x, y)
    assert abs(loss_gpu - loss_ref) <= 1e-3 * loss_ref
    for name, (lo, hi) in {"W1": (sg.OFF_W1, sg.OFF_B1), "b1": (sg.OFF_B1, sg.OFF_W2), "W2": (sg.OFF_W2, sg.OFF_B2),
                           "b2": (sg.OFF_B2, sg.OFF_W3), "W3": (sg.OFF_W3, sg.OFF_B3), "b3": (sg.OFF_B3, sg.OFF_XMU)
                           }.items():
        a, b = g_gpu[lo:hi], g_ref[lo:hi]
        err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        assert err <= 1e-2, (name, err)
    assert np.all(g_gpu[sg.OFF_XMU:] == 0)


@pytest.mark.gpu
@pytest.mark.parametrize("warp_form", [False, True])
def test_inference_kernels_match_oracle(pairs, warp_form):
    _, x, y = pairs
    x = x[:777]
    net = _net(4, x, y)
    got = sg.infer(net, x, warp_form=warp_form)
    want = mo.predict(net, x)
    scale = np.abs(want).max(0)
    assert np.all(np.abs(got - want) <= 1e-2 * scale + 1e-6), np.abs(got - want).max(0) / scale


@pytest.mark.gpu
def test_training_gain(pairs):
    """Training on the tensor cores lowers the held-out error of the
    untrained network by more than 10x on every output (1500 steps of
    2048 samples)."""
    _, x, y = pairs
    xt, yt, xv, yv = x[:5000], y[:5000], x[5000:], y[5000:]
    net = _net(7, xt, yt)
    before = np.sqrt(np.mean((sg.infer(net, xv) - yv) ** 2, axis=0))
    loss = sg.train(net, xt, yt, steps=1500, batch_tiles=16, lr=3e-3, seed=11)
    after = np.sqrt(np.mean((sg.infer(net, xv) - yv) ** 2, axis=0))
    assert loss[-100:].mean() < 0.05 * loss[:10].mean()
    assert np.all(after < before / 10), (before, after)
    # the trained network agrees with the oracle's evaluation of the same weights
    assert np.allclose(sg.infer(net, xv), mo.predict(net, xv), rtol=0, atol=1e-2 * np.abs(yv).max())
