"""Ensembles (icm_ensemble_*): many cases advanced by one launch per
substep over all their active tiles, segments replayed from a CUDA graph.
Each case must end where the same case run alone ends."""
import numpy as np
import pytest

import icempm_b200 as im
from icempm_b200 import configs
from icempm_b200.ensemble import Ensemble

from mpm_cases import compare_states, gpu_model, gpu_state, oracle_run, params, scene

CASES = [  # (cells, seed, overrides)
    ((40, 10), 3, dict(YoungsModulus=8e8, IndVelocity=0.5)),
    ((24, 14), 5, dict(YoungsModulus=2e9, IndVelocity=1.0, DP_phi=50)),
    ((56, 6), 9, dict(IndVelocity=0.2)),
]


def _case(cells, seed, over):
    p = params(**over)
    soa = scene(p, cells=cells, seed=seed, ind_y=0.03, vel=0.05, perturb=5e-4)
    return p, soa


def _alone(p, soa, form, n, rebin):
    m = gpu_model(p, soa, form, tile=1, threads=128)
    m.gpu.set_rebin_interval(rebin)
    m.gpu.run_substeps(m.prms, n)
    hist = m.gpu.force_history(n)
    state = gpu_state(m)
    prms = m.prms.copy()
    m.gpu.close()
    return prms, state, hist


@pytest.mark.gpu
@pytest.mark.parametrize("form", [im.FORM_FP64, im.FORM_FP32])
@pytest.mark.parametrize("graphs", [True, False])
def test_ensemble_matches_cases_run_alone(form, graphs):
    n, rebin = 13, 4
    cases = [_case(*c) for c in CASES]
    ens = Ensemble(form, tile=1, threads=128)
    ens.set(rebin_interval=rebin, graphs=graphs)
    models = []
    for p, soa in cases:
        m = gpu_model(p, soa, form, tile=1, threads=128)
        ens.add(m)
        models.append(m)
    ens.run(n)
    tol_pos, tol = (1e-9, 1e-9) if form == im.FORM_FP64 else (1e-5, 1e-4)
    for (p, soa), m in zip(cases, models):
        got, hist = gpu_state(m), m.gpu.force_history(n)
        q, ref, href = _alone(p, soa, form, n, rebin)
        assert m.prms.SimulationStep == q.SimulationStep and m.prms.SimulationTime == q.SimulationTime
        assert m.prms.indenter_x == q.indenter_x
        err = compare_states(p, got, ref, soa)
        assert err["disp_h"] <= tol_pos and err["strain"] <= tol and err["vel"] <= tol, err
        assert err["crushed_mismatch"] == 0
        scale = max(np.abs(href).max(), 1e-30)
        assert np.abs(hist - href).max() <= 1e3 * tol * scale
        assert m.gpu.error_code == 0
    ens.close()
    for m in models:
        m.gpu.close()


@pytest.mark.gpu
@pytest.mark.parametrize("form", [im.FORM_FP64, im.FORM_FP32])
def test_ensemble_split_tiles_match_cases_run_alone(form):
    """Every measured tile of every case split over two CTAs from the first
    re-binning on: each case still ends where it ends alone."""
    n, rebin = 13, 4
    cases = [_case(*c) for c in CASES]
    ens = Ensemble(form, tile=1, threads=128)
    ens.set(rebin_interval=rebin)
    ens.set_split(4096, 0.0)
    models = []
    for p, soa in cases:
        m = gpu_model(p, soa, form, tile=1, threads=128)
        ens.add(m)
        models.append(m)
    ens.run(n)
    tol_pos, tol = (1e-9, 1e-9) if form == im.FORM_FP64 else (1e-5, 1e-4)
    for (p, soa), m in zip(cases, models):
        got, hist = gpu_state(m), m.gpu.force_history(n)
        _, ref, href = _alone(p, soa, form, n, rebin)
        err = compare_states(p, got, ref, soa)
        assert err["disp_h"] <= tol_pos and err["strain"] <= tol and err["vel"] <= tol, err
        scale = max(np.abs(href).max(), 1e-30)
        assert np.abs(hist - href).max() <= 1e3 * tol * scale
        assert m.gpu.error_code == 0
    ens.close()
    for m in models:
        m.gpu.close()


@pytest.mark.gpu
def test_ensemble_cases_of_different_grids():
    """Cases on grids of different sizes (and so different tile counts) in
    one ensemble each end where they end alone."""
    n, rebin = 11, 4
    specs = [((96, 48), 0.75, (40, 10), 3), ((64, 32), 0.5, (24, 8), 5), ((128, 40), 1.0, (56, 8), 9)]
    cases = []
    for grid, dim, cells, seed in specs:
        p = params(*grid, dim=dim)
        cases.append((p, scene(p, cells=cells, seed=seed, ind_y=0.03, vel=0.05, perturb=5e-4)))
    ens = Ensemble(im.FORM_FP64, tile=1, threads=128)
    ens.set(rebin_interval=rebin)
    models = []
    for p, soa in cases:
        m = gpu_model(p, soa, im.FORM_FP64, tile=1, threads=128)
        ens.add(m)
        models.append(m)
    ens.run(n)
    for (p, soa), m in zip(cases, models):
        got, hist = gpu_state(m), m.gpu.force_history(n)
        _, ref, href = _alone(p, soa, im.FORM_FP64, n, rebin)
        err = compare_states(p, got, ref, soa)
        assert err["disp_h"] <= 1e-9 and err["strain"] <= 1e-9 and err["vel"] <= 1e-9, err
        assert np.abs(hist - href).max() <= 1e-6 * max(np.abs(href).max(), 1e-30)
        assert m.gpu.error_code == 0
    ens.close()
    for m in models:
        m.gpu.close()


@pytest.mark.gpu
def test_ensemble_runs_compose():
    """Two ensemble runs continue each other (a second run re-packs nothing
    and reuses its captured graph)."""
    cases = [_case(*c) for c in CASES[:2]]
    ens = Ensemble(im.FORM_FP32, tile=1, threads=128)
    ens.set(rebin_interval=4)
    models = [gpu_model(p, soa, im.FORM_FP32, tile=1, threads=128) for p, soa in cases]
    for m in models:
        ens.add(m)
    ens.run(9)
    ens.run(9)
    for (p, soa), m in zip(cases, models):
        _, ref, _ = _alone(p, soa, im.FORM_FP32, 18, 4)
        err = compare_states(p, gpu_state(m), ref, soa)
        assert err["disp_h"] <= 1e-5 and err["strain"] <= 1e-4, err
        assert m.prms.SimulationStep == 18
    ens.close()
    for m in models:
        m.gpu.close()


def test_ensemble_argument_errors():
    with pytest.raises(RuntimeError):
        Ensemble(im.FORM_FP64_STEPWISE)
    with pytest.raises(RuntimeError):
        Ensemble(im.FORM_FP32_SURROGATE, tile=1, threads=256)  # the surrogate form's 128-thread limit
    with pytest.raises(RuntimeError):
        Ensemble(im.FORM_FP32, tile=3, threads=32)  # 32x16 tile needs 128 threads


def test_c4_cases():
    cs = configs.c4_cases()
    n = np.array([4 * cx * cy for _, cx, cy, _ in cs])
    assert len(cs) == 64 and n.min() >= 19_000 and n.max() <= 500_000
    assert 7e6 < n.sum() < 1e7
    gx, gy = configs.C4["grid"]
    assert all(cx < gx - 100 and cy < gy - 30 for _, cx, cy, _ in cs)
    phis = [o["DP_phi"] for o, *_ in cs]
    assert 45 <= min(phis) and max(phis) <= 70
    assert cs == configs.c4_cases()  # seeded


def _drifting_block(speed=600.0):
    """A block translating at `speed` m/s: in 120 substeps of 2 us it moves
    0.144 m, 18 cells, further than a 16 x 16 tile."""
    p = params(YoungsModulus=1e9)
    soa = scene(p, cells=(24, 8), seed=11, ind_y=0.03)
    S = im.SoA(soa, p.nPtsPitch, p.nPts)
    room_right = p.GridXDimension - S.pos[0].max()
    S.vel[0] = speed if room_right > 0.3 else -speed
    S.vel[1] = 0.0
    return p, soa


@pytest.mark.gpu
def test_ensemble_flags_mass_outside_active_tiles():
    """Without re-binning the drifting block scatters into tiles its launches
    do not cover: the case's error word gets bit 2. Re-binning every 5
    substeps keeps it covered and the run matches the block run alone."""
    n = 120
    p, soa = _drifting_block()
    ens = Ensemble(im.FORM_FP32, tile=1, threads=128)
    ens.set(rebin_interval=0)
    m = gpu_model(p, soa, im.FORM_FP32, tile=1, threads=128)
    ens.add(m)
    ens.run(n)
    m.gpu.cuda_transfer_from_device()
    m.gpu.synchronize()
    assert m.gpu.error_code & 2
    ens.close()
    m.gpu.close()

    ens = Ensemble(im.FORM_FP32, tile=1, threads=128)
    ens.set(rebin_interval=5)
    m = gpu_model(p, soa, im.FORM_FP32, tile=1, threads=128)
    ens.add(m)
    ens.run(n)
    got = gpu_state(m)
    assert m.gpu.error_code == 0
    _, ref, _ = _alone(p, soa, im.FORM_FP32, n, 5)
    err = compare_states(p, got, ref, soa)
    # float atomics sum in another order in each run (the run alone also
    # splits its heaviest tiles over two CTAs): 18 cells of travel in FP32
    assert err["disp_h"] <= 5e-5 and err["vel"] <= 1e-4, err
    ens.close()
    m.gpu.close()


@pytest.mark.gpu
def test_ensemble_harvest_matches_cases_run_alone():
    """Crushed particles' trial states recorded every second substep inside
    an ensemble are those each case records when run alone."""
    from icempm_b200 import surrogate as sg

    n, every, cap = 6, 2, 200000

    def crushing(seed):
        p = params()
        return p, scene(p, seed=seed, perturb=2e-3, vel=0.05, crushed_frac=0.5, jp_spread=0.005)

    cases = [crushing(3), crushing(8)]
    ens = Ensemble(im.FORM_FP32, tile=1, threads=128)
    models = []
    for p, soa in cases:
        m = gpu_model(p, soa, im.FORM_FP32, tile=1, threads=128)
        sg.set_harvest(m.gpu, cap, every)
        ens.add(m)
        models.append(m)
    ens.run(n)
    for (p, soa), m in zip(cases, models):
        x, y = sg.harvest_pairs(m.gpu, m.prms, cap)
        a = gpu_model(p, soa, im.FORM_FP32, tile=1, threads=128)
        sg.set_harvest(a.gpu, cap, every)
        a.gpu.run_substeps(a.prms, n)
        xa, ya = sg.harvest_pairs(a.gpu, a.prms, cap)
        a.gpu.close()
        assert len(xa) > 1000 and abs(len(x) - len(xa)) <= 0.005 * len(xa)
        k = min(len(x), len(xa))
        for col in range(3):
            u, v = np.sort(x[:, col])[:k], np.sort(xa[:, col])[:k]
            assert np.percentile(np.abs(u - v), 99) <= 1e-3
    ens.close()
    for m in models:
        m.gpu.close()


@pytest.mark.gpu
def test_ensemble_surrogate_form_matches_cases_run_alone():
    """The surrogate form inside an ensemble: each case carries its own
    network, tolerance and counters; each ends close to the same case run
    alone with the same network (accepted predictions may flip near the
    tolerance when float atomics sum in another order)."""
    from icempm_b200 import surrogate as sg

    def crushing(seed):
        p = params()
        return p, scene(p, seed=seed, perturb=2e-3, vel=0.05, crushed_frac=0.5, jp_spread=0.005)

    cases = [crushing(4), crushing(6)]
    h = gpu_model(*cases[0], im.FORM_FP32, tile=1, threads=128)
    sg.set_harvest(h.gpu, 200000, 1)
    h.gpu.run_substeps(h.prms, 10)
    x, y = sg.harvest_pairs(h.gpu, h.prms, 200000)
    h.gpu.close()
    net, _ = sg.fit(x, y, steps=800, batch_tiles=16, lr=3e-3, seed=1)

    n, rebin, tol = 9, 4, 0.05
    ens = Ensemble(im.FORM_FP32_SURROGATE, tile=1, threads=128)
    ens.set(rebin_interval=rebin)
    models = []
    for p, soa in cases:
        m = gpu_model(p, soa, im.FORM_FP32_SURROGATE, tile=1, threads=128)
        sg.set_surrogate(m.gpu, net, tol)
        ens.add(m)
        models.append(m)
    ens.run(n)
    for (p, soa), m in zip(cases, models):
        got = gpu_state(m)
        acc, exact = sg.counts(m.gpu)
        a = gpu_model(p, soa, im.FORM_FP32_SURROGATE, tile=1, threads=128)
        sg.set_surrogate(a.gpu, net, tol)
        a.gpu.set_rebin_interval(rebin)
        a.gpu.run_substeps(a.prms, n)
        ref = gpu_state(a)
        acc_a, exact_a = sg.counts(a.gpu)
        a.gpu.close()
        assert acc > 0 and abs((acc + exact) - (acc_a + exact_a)) <= 0.02 * (acc_a + exact_a), (acc, exact, acc_a, exact_a)
        err = compare_states(p, got, ref, soa)
        G, R = im.SoA(got, p.nPtsPitch, p.nPts), im.SoA(ref, p.nPtsPitch, p.nPts)
        eye = np.array([1.0, 0.0, 0.0, 1.0])[:, None]
        per = np.abs(G.Fe - R.Fe).max(axis=0) / np.abs(R.Fe - eye).max()
        assert err["disp_h"] <= 1e-3, err
        assert np.percentile(per, 99) <= 2e-2, np.percentile(per, 99)
        assert m.gpu.error_code == 0
    ens.close()
    for m in models:
        m.gpu.close()


@pytest.mark.gpu
@pytest.mark.parametrize("form,tol_pos,tol", [(im.FORM_FP64, 1e-9, 1e-9), (im.FORM_FP32, 1e-4, 1e-3)])
def test_ensemble_cases_match_the_oracle(form, tol_pos, tol):
    """Cases of different sizes, grids, materials and indenters in one
    ensemble, each compared with the CPU FP64 oracle directly, over 13
    substeps that cross three re-binnings (every 4 substeps). The states
    carry crushed particles, Jp_inv != 1 and sheared Fe, so every branch of
    the constitutive model runs. Tolerances: FP64 1e-9 (reordered float
    atomics); FP32 1e-4 h in position and 1e-3 of the velocity and strain
    scales."""
    n, rebin = 13, 4
    specs = [((96, 48), 0.75, (40, 10), 3, dict(YoungsModulus=8e8, IndVelocity=0.5)),
             ((64, 32), 0.5, (24, 8), 5, dict(YoungsModulus=2e9, IndVelocity=1.0, DP_phi=50)),
             ((128, 40), 1.0, (56, 8), 9, dict(IndVelocity=0.2, IndDiameter=0.2))]
    cases = []
    for grid, dim, cells, seed, over in specs:
        p = params(*grid, dim=dim, **over)
        cases.append((p, scene(p, cells=cells, seed=seed, ind_y=0.03, vel=0.05, perturb=5e-4, crushed_frac=0.2,
                               jp_spread=0.005)))
    ens = Ensemble(form, tile=1, threads=128)
    ens.set(rebin_interval=rebin)
    models = []
    for p, soa in cases:
        m = gpu_model(p, soa, form, tile=1, threads=128)
        ens.add(m)
        models.append(m)
    ens.run(n)
    for (p, soa), m in zip(cases, models):
        got, hist = gpu_state(m), m.gpu.force_history(n)
        q, ref, _, oerr, href = oracle_run(p, soa, n, threads=4)
        assert oerr == 0 and m.gpu.error_code == 0
        assert m.prms.SimulationStep == q.SimulationStep and m.prms.indenter_x == q.indenter_x
        err = compare_states(p, got, ref, soa)
        assert err["disp_h"] <= tol_pos and err["strain"] <= tol and err["vel"] <= tol, err
        assert err["crushed_mismatch"] <= (0 if form == im.FORM_FP64 else max(2, p.nPts // 1000)), err
        assert err["grain_mismatch"] == 0
        scale = max(np.abs(href).max(), 1e-30)
        assert np.abs(hist - href).max() <= (1e-9 if form == im.FORM_FP64 else 1e-3) * scale
    ens.close()
    for m in models:
        m.gpu.close()
