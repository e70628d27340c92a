"""The CPU FP64 oracle: pinned against the reference's own SVD and against
its committed golden run, plus the invariants of the MLS-MPM transfers."""
import os

import numpy as np
import pytest

import icempm_b200 as im
from oracle import oracle as orc
from tests.mpm_cases import params, scene, oracle_run

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_svd_bit_exact_against_reference_golden():
    g = np.load(os.path.join(GOLDEN, "svd_ref.npz"))
    for A, U, S, V in zip(g["A"], g["U"], g["S"], g["V"]):
        u, s, v = orc.svd2x2(A)
        assert np.array_equal(u, U) and np.array_equal(s, S) and np.array_equal(v, V), A


@pytest.mark.skipif(orc.ref_svd_lib() is None, reason="reference SVD harness not built")
def test_svd_bit_exact_against_reference_binary():
    ref = orc.ref_svd_lib()
    rng = np.random.default_rng(5)
    for k in range(5000):
        A = rng.standard_normal(4) * (10.0 ** rng.integers(-3, 4))
        if k % 3 == 0:
            A = np.array([1.0, 0, 0, 1.0]) + 1e-4 * rng.standard_normal(4)
        A = np.ascontiguousarray(A)
        u, s, v = np.zeros(4), np.zeros(2), np.zeros(4)
        ref.ref_svd(A.ctypes.data, u.ctypes.data, s.ctypes.data, v.ctypes.data)
        U, S, V = orc.svd2x2(A)
        assert np.array_equal(U, u) and np.array_equal(S, s) and np.array_equal(V, v)


def test_svd_reconstructs_and_orders():
    g = np.load(os.path.join(GOLDEN, "svd_ref.npz"))
    for A in g["A"]:
        U, S, V = orc.svd2x2(A)
        Um, Vm = U.reshape(2, 2), V.reshape(2, 2)
        assert np.allclose(Um @ np.diag(S) @ Vm.T, A.reshape(2, 2), atol=1e-13 * (1 + np.abs(A).max()))
        assert S[0] >= S[1]
        assert abs(S[1]) <= abs(S[0]) + 1e-15
        assert np.allclose(Um @ Um.T, np.eye(2), atol=1e-14) and np.linalg.det(Um) == pytest.approx(1.0)


def test_oracle_matches_golden_run():
    g = np.load(os.path.join(GOLDEN, "oracle_small.npz"))
    p = im.SimParams.from_bytes(g["params"].tobytes())
    q, out, bins, err, hist = oracle_run(p, g["soa_in"], 8, threads=1)
    assert np.array_equal(out, g["soa_out"])
    assert np.array_equal(bins, g["bins"]) and np.array_equal(hist, g["hist"])
    assert err == int(g["err"]) and q.to_bytes() == g["params_out"].tobytes()


def test_oracle_thread_count_only_reorders_sums():
    p = params()
    soa = scene(p, perturb=1e-3, vel=0.05, crushed_frac=0.2)
    _, a, ba, _, ha = oracle_run(p, soa, 5, threads=1)
    _, b, bb, _, hb = oracle_run(p, soa, 5, threads=4)
    A = im.SoA(a, p.nPtsPitch, p.nPts)
    B = im.SoA(b, p.nPtsPitch, p.nPts)
    assert np.abs(A.vel - B.vel).max() <= 1e-12 * np.abs(A.vel).max()
    assert np.abs(A.Fe - B.Fe).max() <= 1e-13
    assert np.allclose(ha, hb, rtol=1e-11, atol=1e-9 * np.abs(ha).max())


def test_p2g_conserves_mass_and_momentum():
    p = params()
    soa = scene(p, perturb=1e-3, vel=0.1)
    S = im.SoA(soa, p.nPtsPitch, p.nPts)
    grid = orc.new_grid(p)
    assert orc.p2g(p, soa, grid) == 0
    gp = int(p.nGridPitch)
    m = grid[:gp].sum()
    assert m == pytest.approx(p.nPts * p.ParticleMass, rel=1e-12)
    # APIC and stress terms carry no net momentum: sum_i w_i (x_i - x_p) = 0
    px, py = grid[gp:2 * gp].sum(), grid[2 * gp:3 * gp].sum()
    mv = p.ParticleMass * S.vel.sum(axis=1)
    scale = p.ParticleMass * np.abs(S.vel).sum()
    assert abs(px - mv[0]) < 1e-10 * scale and abs(py - mv[1]) < 1e-10 * scale


def test_update_applies_boundary_conditions_and_gravity():
    p = params()
    gp = int(im.pitch_elems(p.GridTotal))
    p.nGridPitch = gp
    grid = np.zeros(3 * gp)
    rng = np.random.default_rng(0)
    grid[: p.GridTotal] = 1.0
    grid[gp: gp + p.GridTotal] = rng.standard_normal(p.GridTotal) * 1e-3
    grid[2 * gp: 2 * gp + p.GridTotal] = rng.standard_normal(p.GridTotal) * 1e-3
    bins = np.zeros(200)
    orc.update_nodes(p, grid, bins, -10.0, -10.0)
    vx = grid[gp: gp + p.GridTotal].reshape(p.GridY, p.GridX)
    vy = grid[2 * gp: 2 * gp + p.GridTotal].reshape(p.GridY, p.GridX)
    assert np.all(vx[:3] == 0) and np.all(vy[:3] == 0)          # sticky floor
    assert np.all(vy[-3:] <= 0)                                    # top wall
    assert np.all(vx[:, :3] >= 0) and np.all(vx[:, -3:] <= 0)      # side walls
    assert np.all(bins == 0)


def test_indenter_contact_removes_inward_velocity_and_bins_force():
    p = params()
    gp = int(im.pitch_elems(p.GridTotal))
    p.nGridPitch = gp
    grid = np.zeros(3 * gp)
    grid[: p.GridTotal] = 2.0
    ix, iy = 0.4, 0.3                       # centre of the cylinder
    bins = np.zeros(200)
    tot = orc.update_nodes(p, grid, bins, ix, iy)
    h = p.cellsize
    X, Y = np.meshgrid(np.arange(p.GridX) * h, np.arange(p.GridY) * h)
    inside = (X - ix) ** 2 + (Y - iy) ** 2 < p.IndRSq
    vx = grid[gp: gp + p.GridTotal].reshape(p.GridY, p.GridX)
    # nodes at rest inside the cylinder moving at +0.2 m/s in x: those on its
    # leading (right) half are pushed, the rest keep their velocity
    lead = inside & (X > ix)
    assert np.all(vx[lead] > 0)
    assert bins.sum() != 0 and np.allclose([bins[0::2].sum(), bins[1::2].sum()], tot)
    assert tot[0] < 0                       # reaction opposes the motion
