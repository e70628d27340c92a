"""The oracle against the reference's own code.

oracle/build_ref.sh compiles lines 1-416 of the reference's
simulation/gpu_implementation5.cu -- KirchhoffStress_Wolper, ComputePQ,
Wolper_Drucker_Prager, GetParametersForGrain,
CheckIfPointIsInsideFailureSurface, the SVD glue and the bodies of
v2_kernel_p2g, v2_kernel_update_nodes and v2_kernel_g2p -- for the host into
oracle/_ref/libref_step.so (an Eigen-subset stub stands in for Eigen, host
variables for threadIdx/blockIdx, a plain addition for atomicAdd). These
tests hold the oracle (oracle/mpm_oracle.c) to that library bit for bit:
per function over every branch, and per substep (Model::Step's loop,
model.cpp:20-29) on scenes whose stencils stay inside the grid, including
the 69,632-particle 512x128 workload over 100 substeps. The force bins are summed in a
different order (the oracle adds each substep's sum to the bins, the
reference adds node by node) and agree to 1e-14 relative.
"""
import ctypes as C

import numpy as np
import pytest

import icempm_b200 as im
from icempm_b200 import configs
from oracle import oracle as orc
from tests.mpm_cases import params, scene

REF = orc.ref_step_lib()
pytestmark = pytest.mark.skipif(REF is None, reason="oracle/_ref/libref_step.so not built (no reference checkout)")


def _ref_constitutive(p, F, jp, crushed, grain):
    F = np.ascontiguousarray(F, dtype=np.float64).reshape(4).copy()
    j = np.array([jp])
    c = np.array([crushed], dtype=np.uint8)
    pq = np.zeros(2)
    REF.ref_constitutive(C.byref(p), F.ctypes.data, j.ctypes.data, c.ctypes.data, int(grain), pq[:1].ctypes.data,
                         pq[1:].ctypes.data)
    return F, float(j[0]), int(c[0]), float(pq[0]), float(pq[1])


def _strains(rng, n):
    """Deformation gradients over the regimes the substep meets: small
    strains, shear, tension, compression past the crushing pressure,
    inverted and nearly degenerate states, and rotations of each."""
    out = []
    for k in range(n):
        kind = k % 7
        if kind == 0:
            F = np.eye(2) + 1e-4 * rng.standard_normal((2, 2))
        elif kind == 1:
            F = np.eye(2) + 1e-2 * rng.standard_normal((2, 2))
        elif kind == 2:
            F = np.diag(rng.uniform(1.0, 1.3, 2)) + 1e-3 * rng.standard_normal((2, 2))   # tension
        elif kind == 3:
            F = np.diag(rng.uniform(0.6, 0.95, 2)) + 1e-3 * rng.standard_normal((2, 2))  # compression
        elif kind == 4:
            s = rng.uniform(0.9, 1.1)
            F = s * np.eye(2) + 1e-9 * rng.standard_normal((2, 2))                    # near-degenerate
        elif kind == 5:
            F = np.diag([1.05, -0.2]) + 1e-3 * rng.standard_normal((2, 2))            # inverted
        else:
            F = np.array([[1.0, rng.uniform(-0.3, 0.3)], [0.0, 1.0]])                 # simple shear
        th = rng.uniform(-np.pi, np.pi)
        R = np.array([[np.cos(th), -np.sin(th)], [np.sin(th), np.cos(th)]])
        out.append((R @ F).reshape(4) if k % 2 else F.reshape(4))
    return out


def test_parameter_block_is_the_reference_layout():
    assert REF.ref_params_size() == C.sizeof(im.SimParams) == 432


def test_kirchhoff_bit_exact():
    p = params()
    rng = np.random.default_rng(1)
    for F in _strains(rng, 3000):
        F = np.ascontiguousarray(F)
        t = np.zeros(4)
        REF.ref_kirchhoff(C.byref(p), F.ctypes.data, t.ctypes.data)
        assert np.array_equal(orc.kirchhoff(p, F), t), F


def test_compute_pq_bit_exact():
    p = params()
    rng = np.random.default_rng(2)
    for F in _strains(rng, 3000):
        F = np.ascontiguousarray(F)
        r = np.zeros(17)
        REF.ref_compute_pq(C.byref(p), F.ctypes.data, r.ctypes.data)
        assert np.array_equal(orc.compute_pq(p, F), r), F


def test_grain_parameters_bit_exact():
    p = params()
    for g in list(range(-40, 700)) + [32767, -32768]:
        r = np.zeros(5)
        REF.ref_grain_params(C.byref(p), g, r.ctypes.data)
        assert np.array_equal(orc.grain_params(p, g), r), g


def test_failure_check_every_branch():
    p = params()
    rng = np.random.default_rng(3)
    seen = set()
    for k in range(20000):
        g = int(rng.integers(0, 600))
        pmin, pmax, qmax, beta, msq = orc.grain_params(p, g)
        region = k % 3
        if region == 0:
            pt = -rng.uniform(3e6, 3e7)                       # below the tension cut-off
        elif region == 1:
            pt = -rng.uniform(0, 3e6)                         # tension cap
        else:
            pt = rng.uniform(0, 1.2 * pmax)                   # NACC ellipse
        qt = rng.uniform(0, 1.5 * qmax)
        want = REF.ref_failure_check(C.byref(p), g, pt, qt)
        assert orc.failure_check(p, g, pt, qt) == want, (g, pt, qt)
        seen.add((region, want))
    # both outcomes on the tension cap and the ellipse, crushing below the cut-off
    assert {(0, 1), (1, 0), (1, 1), (2, 0), (2, 1)} <= seen


def test_constitutive_update_every_branch():
    p = params()
    rng = np.random.default_rng(4)
    seen = set()
    for k, F in enumerate(_strains(rng, 6000)):
        crushed = int(k % 3 != 0)
        jp = 1.0 + (0.02 * rng.standard_normal() if k % 5 else -0.01)
        g = int(rng.integers(0, 400))
        got = orc.constitutive(p, F, jp, crushed, g)
        want = _ref_constitutive(p, F, jp, crushed, g)
        assert np.array_equal(got[0], want[0]) and got[1:] == want[1:], (F, jp, crushed, g)
        # which branch of Wolper_Drucker_Prager ran (gpu_implementation5.cu:59-92)
        _, _, cr, pt, qt = want
        if cr:
            if pt < -p.DP_threshold_p or jp < 1:
                seen.add("hydrostatic")
            elif pt > p.IceCompressiveStrength:
                seen.add("q=0")
            else:
                q1 = min((pt + p.DP_threshold_p) * p.DP_tan_phi, p.IceShearStrength)
                seen.add("project" if qt >= q1 else "inside")
        else:
            seen.add("intact")
    assert {"hydrostatic", "q=0", "project", "inside", "intact"} <= seen


def _ref_run(p, soa, n):
    q = p.copy()
    s = soa.copy()
    grid = np.zeros(3 * int(q.nGridPitch))
    bins = np.zeros(2 * q.n_indenter_subdivisions)
    err = REF.ref_run_substeps(C.byref(q), s.ctypes.data, grid.ctypes.data, bins.ctypes.data, n)
    return q, s, bins, err


def _oracle_run(p, soa, n):
    q = p.copy()
    s = soa.copy()
    grid = orc.new_grid(q)
    bins = np.zeros(2 * q.n_indenter_subdivisions)
    err, _ = orc.run_substeps(q, s, grid, bins, n, threads=1, history=False)
    return q, s, bins, err


def _assert_same_run(p, soa, n):
    qa, a, ba, ea = _oracle_run(p, soa, n)
    qb, b, bb, eb = _ref_run(p, soa, n)
    assert ea == eb == 0
    assert np.array_equal(a, b), "particle SoA differs from the reference's own kernels"
    assert qa.SimulationStep == qb.SimulationStep and qa.SimulationTime == qb.SimulationTime
    assert qa.indenter_x == qb.indenter_x
    scale = max(np.abs(bb).max(), 1e-300)
    assert np.abs(ba - bb).max() <= 1e-14 * scale
    return a


def test_substeps_bit_exact_with_every_branch():
    # perturbed strains, velocities, 30 % crushed and Jp_inv spread: every
    # constitutive branch, indenter contact, the frame boundary (recordPQ)
    p = params(96, 48, dim=0.75, dt=2e-6)
    p.UpdateEveryNthStep = 4
    soa = scene(p, cells=(48, 12), seed=9, ind_y=0.05, perturb=3e-3, vel=0.05, crushed_frac=0.3, jp_spread=0.01)
    out = _assert_same_run(p, soa, 9)
    S = im.SoA(out, p.nPtsPitch, p.nPts)
    assert S.crushed.sum() > 0 and np.abs(S.P).max() > 0


def test_substeps_bit_exact_on_the_70k_workload():
    # 69,632 particles on the 512x128 grid (dt 2e-6), the indenter touching
    # the block's left face: 100 substeps with contact forces every substep
    p, soa = configs.make_scene("c1_70k")
    _assert_same_run(p, soa, 100)
    q, _, bins, _ = _ref_run(p, soa, 1)
    assert np.abs(bins).max() > 0
