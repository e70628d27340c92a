"""The surrogate form of the substep (FORM_FP32_SURROGATE): training data
harvested from the FP32 form and labelled by the exact projection, the
form's exact fallback, and a trained network inside the substep."""
import numpy as np
import pytest

import icempm_b200 as im
from icempm_b200 import surrogate as sg
from oracle import mlp_oracle as mo

from mpm_cases import compare_states, gpu_model, gpu_state, params, scene


def _crushing_case():
    p = params()
    soa = scene(p, perturb=2e-3, vel=0.05, crushed_frac=0.5, jp_spread=0.005)
    return p, soa


def _run(p, soa, form, n, net=None, tol=0.02, harvest=0):
    # the surrogate form runs 128-thread blocks (its per-warp scratch)
    m = gpu_model(p, soa, form, threads=128)
    if net is not None:
        sg.set_surrogate(m.gpu, net, tol)
    if harvest:
        sg.set_harvest(m.gpu, harvest, 1)
    m.gpu.run_substeps(m.prms, n)
    return m, gpu_state(m)


def _pairs_from_gpu(n_substeps=20, cap=200000):
    p, soa = _crushing_case()
    m, _ = _run(p, soa, im.FORM_FP32, n_substeps, harvest=cap)
    x, y = sg.harvest_pairs(m.gpu, m.prms, cap)
    m.gpu.close()
    return p, x, y


@pytest.mark.gpu
def test_harvested_labels_match_oracle():
    """Pairs recorded from the FP32 form and labelled on the GPU agree with
    the CPU restatement of the projection applied to the same features."""
    p, x, y = _pairs_from_gpu(n_substeps=4)
    assert len(x) > 1000
    m = mo.material(p)
    assert np.allclose(x[:, 3], m["kappa"] * 1e-9) and np.allclose(x[:, 5], m["qmax"] * 1e-7)
    idx = np.random.default_rng(0).choice(len(x), min(2000, len(x)), replace=False)
    bad = 0
    for i in idx:
        s0, s1, jp = 1.0 + x[i, 0] / 1e3, 1.0 + x[i, 1] / 1e3, 1.0 + x[i, 2] / 1e2
        _, s0n, s1n, jpn = mo.dp_project(m["kappa"], m["mu"], m["p_thr"], m["tan_phi"], m["pmax"], m["qmax"], s0, s1, jp)
        want = mo.targets(s0, s1, jp, s0n, s1n, jpn)
        bad += not np.allclose(y[i], want, rtol=0, atol=2e-3)
    # features are stored in FP32: a state within rounding of a branch
    # boundary may label differently
    assert bad <= 0.01 * len(idx), bad


@pytest.mark.gpu
def test_surrogate_form_with_exact_fallback_matches_fp32_form():
    """With a tolerance nothing can meet, every crushed particle takes the
    exact projection: the surrogate form is then the FP32 form."""
    p, soa = _crushing_case()
    net = sg.init_net(3)
    m_s, got = _run(p, soa, im.FORM_FP32_SURROGATE, 12, net=net, tol=1e-30)
    acc, exact = sg.counts(m_s.gpu)
    m_s.gpu.close()
    m_f, ref = _run(p, soa, im.FORM_FP32, 12)
    m_f.gpu.close()
    assert acc == 0 and exact > 1000
    err = compare_states(p, got, ref, soa)
    assert err["disp_h"] <= 1e-5 and err["strain"] <= 1e-4 and err["vel"] <= 1e-4, err
    assert err["crushed_mismatch"] == 0


@pytest.mark.gpu
def test_trained_surrogate_in_the_substep():
    """A network trained on harvested pairs runs inside the substep: a
    quarter or more of all crushed-particle updates take the network's
    projection (the hydrostatic branch, about half of them in this scene
    with Jp_inv spread around 1, is always the closed form), and the state
    stays close to the FP32 form's."""
    p, x, y = _pairs_from_gpu(n_substeps=30)
    net, loss = sg.fit(x, y, steps=1500, batch_tiles=32, lr=3e-3, seed=5)
    assert loss[-50:].mean() < 0.05 * loss[:5].mean()
    p, soa = _crushing_case()
    m_s, got = _run(p, soa, im.FORM_FP32_SURROGATE, 30, net=net, tol=0.05)
    acc, exact = sg.counts(m_s.gpu)
    m_s.gpu.close()
    m_f, ref = _run(p, soa, im.FORM_FP32, 30)
    m_f.gpu.close()
    assert acc >= 0.25 * (acc + exact), (acc, exact)
    err = compare_states(p, got, ref, soa)
    # accepted predictions differ from the exact map within the tolerance,
    # and over 30 substeps a few particles near a branch boundary take the
    # other branch: the bulk is bounded tightly, the worst particle loosely
    G, R = im.SoA(got, p.nPtsPitch, p.nPts), im.SoA(ref, p.nPtsPitch, p.nPts)
    eye = np.array([1.0, 0.0, 0.0, 1.0])[:, None]
    per = np.abs(G.Fe - R.Fe).max(axis=0) / np.abs(R.Fe - eye).max()
    assert err["disp_h"] <= 1e-3, err
    assert np.percentile(per, 99) <= 2e-2 and per.max() <= 0.5, (np.percentile(per, 99), per.max())


@pytest.mark.gpu
def test_surrogate_form_needs_a_network():
    p, soa = _crushing_case()
    m = gpu_model(p, soa, im.FORM_FP32_SURROGATE, threads=128)
    with pytest.raises(RuntimeError, match="without a network"):
        m.gpu.run_substeps(m.prms, 2)
    sg.set_surrogate(m.gpu, sg.init_net(0))
    m.gpu.set_tile(1, 256)
    with pytest.raises(RuntimeError, match="at most 128 threads"):
        m.gpu.run_substeps(m.prms, 2)
    m.gpu.close()
