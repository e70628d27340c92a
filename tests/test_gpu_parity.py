"""Parity of the CUDA substep against the CPU FP64 oracle, through the C ABI.

Tolerances (relative to the scale of each reference field):
  FP64 forms   1e-9  (float atomics reorder sums: ~1e-16 per sum, grown by
               the dynamics over the substeps compared), crushed flags equal;
  FP32 form    one substep from a perturbed state: velocity 1e-4, strain
               Fe - I 1e-4 (on particles whose crushed flag agrees; a
               threshold decision may flip on a few), force 1e-4;
               200 substeps of indentation: positions within 1e-3 h,
               velocity and strain 1e-2, peak force 1e-2.
"""
import numpy as np
import pytest

import icempm_b200 as im
from oracle import oracle as orc
from tests.mpm_cases import params, scene, gpu_model, gpu_state, oracle_run, compare_states, max_rel

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-9


def perturbed_case(seed=7, grid=(96, 48), cells=(48, 12), shift_x=0.0):
    p = params(*grid, dim=0.75, dt=2e-6)
    soa = scene(p, cells=cells, seed=seed, ind_y=0.05, perturb=3e-3, vel=0.05, crushed_frac=0.3, jp_spread=0.01,
                shift_x=shift_x)
    return p, soa


def test_stepwise_kernels_one_by_one():
    p, soa = perturbed_case()
    m = gpu_model(p, soa, im.FORM_FP64_STEPWISE)
    g = m.gpu
    grid = orc.new_grid(p)
    assert orc.p2g(p, soa, grid) == 0
    g.cuda_reset_grid()
    g.cuda_p2g()
    gg = g.grid_from_device()
    gp = int(p.nGridPitch)
    for r in range(3):
        assert max_rel(gg[r * gp:(r + 1) * gp], grid[r * gp:(r + 1) * gp]) < 1e-13, r
    # update from the oracle's grid on both sides
    g.grid_to_device(grid)
    g.cuda_reset_indenter_force_accumulator()
    ix = p.indenter_x + 0.03
    g.cuda_update_nodes(ix, p.indenter_y)
    bins = np.zeros(200)
    orc.update_nodes(p, grid, bins, ix, p.indenter_y)
    gg = g.grid_from_device()
    assert np.abs(gg - grid).max() <= 1e-13 * np.abs(grid).max()
    g.cuda_transfer_from_device()
    g.synchronize()
    assert bins.any() and max_rel(g.host_side_indenter_force_accumulator, bins) < 1e-12
    # G2P from the same grid
    ref = soa.copy()
    orc.g2p(p, ref, grid, True)
    g.grid_to_device(grid)
    g.cuda_g2p(True)
    got = gpu_state(m)
    e = compare_states(p, got, ref, soa)
    assert e["crushed_mismatch"] == 0 and e["grain_mismatch"] == 0
    assert max(e["disp_rel"], e["vel"], e["strain"], e["Bp"]) < 1e-12, e
    G, R = im.SoA(got, p.nPtsPitch, p.nPts), im.SoA(ref, p.nPtsPitch, p.nPts)
    assert max_rel(G.P, R.P) < 1e-10 and max_rel(G.Q, R.Q) < 1e-10


@pytest.mark.parametrize("form,tile", [(im.FORM_FP64_STEPWISE, 1), (im.FORM_FP64, 0), (im.FORM_FP64, 1),
                                       (im.FORM_FP64, 2), (im.FORM_FP64, 3)])
@pytest.mark.parametrize("n", [1, 12])
def test_fp64_forms_match_oracle(form, tile, n):
    p, soa = perturbed_case()
    m = gpu_model(p, soa, form, tile)
    m.gpu.run_substeps(m.prms, n)
    got = gpu_state(m)
    q, ref, bins, err, hist = oracle_run(p, soa, n)
    e = compare_states(p, got, ref, soa)
    print(im.FORM_NAMES[form], tile, n, e)
    assert e["crushed_mismatch"] == 0 and e["grain_mismatch"] == 0
    assert max(e["disp_rel"], e["vel"], e["strain"], e["Bp"], e["Jp"]) < FP64_TOL, e
    assert max_rel(m.gpu.force_history(n), hist) < FP64_TOL
    assert max_rel(m.gpu.host_side_indenter_force_accumulator, bins) < FP64_TOL
    assert m.gpu.error_code == err == 0
    assert m.prms.SimulationStep == q.SimulationStep and m.prms.SimulationTime == q.SimulationTime
    assert m.prms.indenter_x == q.indenter_x


FP32_FORMS = [im.FORM_FP32, im.FORM_FP32_COMPENSATED]


@pytest.mark.parametrize("form", FP32_FORMS)
@pytest.mark.parametrize("tile", [0, 1, 3])
def test_fp32_one_substep_all_branches(tile, form):
    """One substep from a perturbed state (crushed particles, Jp_inv != 1,
    sheared Fe): every branch of the FP32 strain form (plain and with
    compensated per-cell momentum sums) against the oracle."""
    p = params(96, 48, dim=0.75, dt=2e-6)
    soa = scene(p, cells=(48, 12), seed=5, ind_y=0.05, perturb=2e-2, vel=0.05, crushed_frac=0.5, jp_spread=0.02)
    m = gpu_model(p, soa, form, tile)
    m.gpu.run_substeps(m.prms, 1)
    got = gpu_state(m)
    q, ref, bins, err, hist = oracle_run(p, soa, 1)
    e = compare_states(p, got, ref, soa)
    n = p.nPts
    print(im.FORM_NAMES[form], "1 substep", tile, e, "redo", m.gpu.fp64_redo_count(),
          "crushed", int(im.SoA(ref, p.nPtsPitch, n).crushed.sum()))
    assert e["crushed_mismatch"] <= max(2, n // 1000)
    assert e["grain_mismatch"] == 0
    assert e["vel"] < 1e-4 and e["Bp"] < 1e-3 and e["disp_h"] < 1e-5, e
    G, R = im.SoA(got, p.nPtsPitch, n), im.SoA(ref, p.nPtsPitch, n)
    same = G.crushed == R.crushed
    eye = np.array([1.0, 0, 0, 1.0])[:, None]
    strain = np.abs((G.Fe - eye) - (R.Fe - eye))[:, same].max() / np.abs(R.Fe - eye).max()
    assert strain < 1e-4, strain
    assert max_rel(m.gpu.force_history(1), hist) < 1e-4


@pytest.mark.parametrize("form", FP32_FORMS)
@pytest.mark.parametrize("tile", [1, 3])
def test_fp32_indentation_tracks_oracle(tile, form):
    """200 substeps of a block pushed by the indenter (smooth state): the FP32
    forms stay within 1e-3 h of the FP64 oracle."""
    p = params(96, 48, dim=0.75, dt=2e-6)
    soa = scene(p, cells=(48, 12), seed=3, ind_y=0.05)
    S = im.SoA(soa, p.nPtsPitch, p.nPts)
    p.indenter_x = p.indenter_x_initial = S.pos[0].min() - 0.15 + 2 * p.cellsize  # 2 cells of overlap
    n = 200
    m = gpu_model(p, soa, form, tile)
    m.gpu.run_substeps(m.prms, n)
    got = gpu_state(m)
    q, ref, bins, err, hist = oracle_run(p, soa, n, threads=4)
    e = compare_states(p, got, ref, soa)
    fh = m.gpu.force_history(n)
    f_ref = np.hypot(hist[:, 0], hist[:, 1])
    f_got = np.hypot(fh[:, 0], fh[:, 1])
    peak = abs(f_got.max() - f_ref.max()) / f_ref.max()
    print(im.FORM_NAMES[form], "indentation", tile, e, "peak force", peak, "redo", m.gpu.fp64_redo_count())
    assert f_ref.max() > 0
    assert e["disp_h"] < 1e-3 and e["vel"] < 1e-2 and e["strain"] < 1e-2, e
    assert peak < 1e-2
    assert e["grain_mismatch"] == 0


def test_out_of_grid_raises_error_flag():
    p = params(96, 48, dim=0.75, dt=2e-6)
    soa = scene(p, cells=(48, 12), seed=2)
    S = im.SoA(soa, p.nPtsPitch, p.nPts)
    S.pos[0, 5] = 0.2 * p.cellsize          # stencil reaches node -1? no: truncation keeps base 0
    S.pos[0, 7] = (p.GridX - 1.2) * p.cellsize  # stencil leaves the grid on the right
    for form in (im.FORM_FP64_STEPWISE, im.FORM_FP64, im.FORM_FP32):
        m = gpu_model(p, soa, form)
        m.gpu.run_substeps(m.prms, 1)
        gpu_state(m)
        _, _, _, err, _ = oracle_run(p, soa, 1)
        assert err == 1 and m.gpu.error_code == 1, form


def test_ragged_grid_and_empty_tiles():
    p = params(70, 37, dim=0.75 * 70 / 96, dt=2e-6)
    soa = scene(p, cells=(30, 9), seed=9, ind_y=0.04, perturb=2e-3, vel=0.05, crushed_frac=0.2)
    q, ref, bins, err, hist = oracle_run(p, soa, 6)
    for tile in range(4):
        m = gpu_model(p, soa, im.FORM_FP64, tile)
        m.gpu.run_substeps(m.prms, 6)
        e = compare_states(p, gpu_state(m), ref, soa)
        assert e["crushed_mismatch"] == 0 and max(e["disp_rel"], e["vel"], e["strain"]) < FP64_TOL, (tile, e)


@pytest.mark.parametrize("grid", [(1536, 1152), (2304, 1024)])
def test_many_tiles(grid):
    """Grids of 6,912 tiles of 16x16 cells (the tile sort's shared memory
    above 48 KB) and of 9,216 tiles (beyond the sort's limit: launched in
    tile order), re-binned every 3 substeps so that the sort runs on
    measured costs, against the oracle."""
    gx, gy = grid
    p = params(gx, gy, dim=0.75 * gx / 96, dt=2e-6)
    soa = scene(p, cells=(48, 12), seed=5, ind_y=0.05, perturb=2e-3, vel=0.05, crushed_frac=0.2)
    q, ref, bins, err, hist = oracle_run(p, soa, 7)
    for form in (im.FORM_FP64, im.FORM_FP32):
        m = gpu_model(p, soa, form, 1, 128)
        m.gpu.set_rebin_interval(3)
        m.gpu.run_substeps(m.prms, 7)
        e = compare_states(p, gpu_state(m), ref, soa)
        tol = FP64_TOL if form == im.FORM_FP64 else 1e-3
        assert m.gpu.error_code == 0 and max(e["disp_rel"], e["vel"], e["strain"]) < tol, (grid, form, e)
        if form == im.FORM_FP64:
            assert e["crushed_mismatch"] == 0, e


def test_zero_particles():
    p = params(64, 32, dim=0.5, dt=2e-6)
    soa = scene(p, cells=(8, 4), seed=1)
    for form in (im.FORM_FP64_STEPWISE, im.FORM_FP64, im.FORM_FP32):
        m = gpu_model(p, soa, form)
        m.prms.nPts = 0
        m.gpu.run_substeps(m.prms, 3)
        gpu_state(m)
        assert m.prms.SimulationStep == 3 and m.gpu.error_code == 0


@pytest.mark.parametrize("form", [im.FORM_FP64, im.FORM_FP32])
def test_runs_compose(form):
    """Two calls of 5 substeps equal one call of 10 (state round-trips
    through the reference layout between calls)."""
    p, soa = perturbed_case(seed=4)
    a = gpu_model(p, soa, form)
    a.gpu.run_substeps(a.prms, 10)
    sa = gpu_state(a)
    b = gpu_model(p, soa, form)
    b.gpu.run_substeps(b.prms, 5)
    gpu_state(b)
    b.gpu.run_substeps(b.prms, 5)
    sb = gpu_state(b)
    e = compare_states(p, sb, sa, soa)
    tol = FP64_TOL if form == im.FORM_FP64 else 1e-4
    assert e["crushed_mismatch"] == 0 and max(e["disp_rel"], e["vel"], e["strain"]) < tol, e


def test_model_step_runs_one_frame():
    """icy::Model::Step: frame of UpdateEveryNthStep substeps, bins reset per
    frame, P/Q recorded on the frame's last substep (model.cpp:11-47)."""
    p, soa = perturbed_case(seed=8)
    for form in (im.FORM_FP64_STEPWISE, im.FORM_FP64):
        m = gpu_model(p, soa, form)
        m.prms.UpdateEveryNthStep = 7
        assert m.Step()
        m.gpu.synchronize()
        got = m.gpu.tmp_transfer_buffer.copy()
        q = p.copy()
        q.UpdateEveryNthStep = 7
        _, ref, bins, err, hist = oracle_run(q, soa, 7)
        e = compare_states(p, got, ref, soa)
        assert m.prms.SimulationStep == 7 and max(e["vel"], e["strain"]) < FP64_TOL
        G, R = im.SoA(got, p.nPtsPitch, p.nPts), im.SoA(ref, p.nPtsPitch, p.nPts)
        assert max_rel(G.P, R.P) < FP64_TOL and max_rel(G.Q, R.Q) < FP64_TOL
        assert max_rel(m.gpu.host_side_indenter_force_accumulator, bins) < FP64_TOL
        # second frame: bins restart from zero
        assert m.Step()
        m.gpu.synchronize()
        assert m.prms.SimulationStep == 14


@pytest.mark.parametrize("form", [im.FORM_FP64, im.FORM_FP32])
@pytest.mark.parametrize("tile", [0, 1, 3])
def test_split_tiles_keep_parity(form, tile):
    """Every tile with a measured cost run as two CTAs (one per half of its
    cell groups) from the first re-binning on: results match the oracle as
    without splitting, reaction force included (only the first half adds
    it)."""
    p, soa = perturbed_case(seed=14)
    n = 12
    m = gpu_model(p, soa, form, tile, 128)
    m.gpu.set_rebin_interval(3)
    m.gpu.set_tile_split(4096, 0.0)
    m.gpu.run_substeps(m.prms, n)
    got = gpu_state(m)
    q, ref, bins, err, hist = oracle_run(p, soa, n)
    e = compare_states(p, got, ref, soa)
    if form == im.FORM_FP64:
        assert e["crushed_mismatch"] == 0 and max(e["disp_rel"], e["vel"], e["strain"], e["Bp"]) < FP64_TOL, e
        assert max_rel(m.gpu.force_history(n), hist) < FP64_TOL
    else:
        assert e["disp_h"] < 1e-4 and e["vel"] < 5e-3, e
        assert max_rel(m.gpu.force_history(n), hist) < 1e-2
    assert e["grain_mismatch"] == 0
    assert m.gpu.error_code == 0


@pytest.mark.parametrize("form", [im.FORM_FP64, im.FORM_FP32])
def test_rebinning_keeps_parity(form):
    """Re-binning the particles between substeps changes only their order:
    results match the oracle as without it."""
    p, soa = perturbed_case(seed=12)
    n = 12
    m = gpu_model(p, soa, form, 1, 128)
    m.gpu.set_rebin_interval(3)
    m.gpu.run_substeps(m.prms, n)
    got = gpu_state(m)
    q, ref, bins, err, hist = oracle_run(p, soa, n)
    e = compare_states(p, got, ref, soa)
    if form == im.FORM_FP64:
        assert e["crushed_mismatch"] == 0 and max(e["disp_rel"], e["vel"], e["strain"], e["Bp"]) < FP64_TOL, e
        assert max_rel(m.gpu.force_history(n), hist) < FP64_TOL
    else:
        assert e["disp_h"] < 1e-4 and e["vel"] < 5e-3, e
    assert e["grain_mismatch"] == 0


@pytest.mark.parametrize("form", [im.FORM_FP64, im.FORM_FP32])
def test_emptied_tile_next_to_the_indenter_is_not_split(form):
    """A strip of particles starts in the second column of 16x8 tiles and
    moves left at 400 m/s into the first, so the tile it leaves keeps a
    measured cost while it holds no particles (from substep 20 on). Its
    first node columns still get mass from the strip's stencils, and the
    indenter touches them. With
    every measured tile split (ratio 0) and a re-binning every 2 substeps,
    the emptied tile must run whole: its reaction force counts once, and the
    force history matches the oracle."""
    p = params(96, 48, dim=0.75, dt=2e-6, IndDiameter=0.02)
    soa = scene(p, cells=(2, 6), seed=31, ind_y=0.03)
    S = im.SoA(soa, p.nPtsPitch, p.nPts)
    h = p.cellsize
    S.pos[0] += 16.6 * h - S.pos[0].min()      # bases 16 and 17: the second tile column
    S.pos[1] += 8.3 * h - S.pos[1].min()       # tile row 1 (y cells 8..13; stencils reach node row 15)
    S.vel[0] = -400.0
    S.vel[1] = 0.0
    S.Bp[:] = 0.0
    # above the strip: it touches node row 15 of the emptied tile without stopping the strip
    p.indenter_x = p.indenter_x_initial = 16.5 * h
    p.indenter_y = p.indenter_y_initial = 15.6 * h
    n = 30
    m = gpu_model(p, soa, form, 0, 128)
    m.gpu.set_rebin_interval(2)
    m.gpu.set_tile_split(4096, 0.0)
    m.gpu.run_substeps(m.prms, n)
    got = gpu_state(m)
    fh = m.gpu.force_history(n)
    q, ref, bins, err, hist = oracle_run(p, soa, n)
    R = im.SoA(ref, p.nPtsPitch, p.nPts)
    assert (R.pos[0] / h - 0.5).astype(int).max() <= 15   # the strip has left the second tile
    assert np.abs(hist[-10:]).max() > 0                   # and the indenter still pushes it
    e = compare_states(p, got, ref, soa)
    if form == im.FORM_FP64:
        assert max(e["disp_rel"], e["vel"], e["strain"]) < FP64_TOL, e
        assert max_rel(fh, hist) < FP64_TOL
    else:
        assert e["disp_h"] < 1e-4 and e["vel"] < 5e-3, e
        assert max_rel(fh, hist) < 1e-2
    assert m.gpu.error_code == 0
