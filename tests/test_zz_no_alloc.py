"""The substep entry point that allocates nothing (icm_run_substeps_noalloc).

It serves callers that cannot allocate device memory while they run (an
allocation can block or synchronise the device, or another allocator owns
the GPU's memory). Its grid scratch is a fixed array inside the library, so
this test checks, through the C ABI, that two calls in a row give what the
allocating entry point gives on the same input, and what the CPU oracle
gives on the 69,632-particle 512x128 workload, within the FP64 tolerance of
the other parity tests (1e-9), and that an oversized grid is refused.
"""
import ctypes as C

import numpy as np
import pytest

import icempm_b200 as im
from tests.mpm_cases import params, scene, gpu_model, gpu_state, compare_states, max_rel

pytestmark = pytest.mark.gpu

TOL = 1e-9


def _noalloc():
    L = im.library()
    f = L.icm_run_substeps_noalloc
    f.restype = C.c_int
    f.argtypes = [C.POINTER(im.SimParams), C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    return f


def test_noalloc_matches_allocating_entry_point_twice():
    import torch

    p = params(96, 48, dim=0.75, dt=2e-6)
    soa = scene(p, cells=(48, 12), seed=21, ind_y=0.05, perturb=3e-3, vel=0.05, crushed_frac=0.3, jp_spread=0.01)
    n = 4

    # the allocating entry point, two calls
    m = gpu_model(p, soa, im.FORM_FP64_STEPWISE)
    m.gpu.cuda_reset_indenter_force_accumulator()
    m.gpu.run_substeps(m.prms, n)
    m.gpu.run_substeps(m.prms, n)
    ref = gpu_state(m)
    ref_bins = m.gpu.host_side_indenter_force_accumulator.copy()
    ref_params = m.prms.copy()
    m.gpu.close()

    # the entry point without allocation, on caller-owned device buffers
    f = _noalloc()
    q = p.copy()
    pts = torch.tensor(soa, dtype=torch.float64, device="cuda")
    bins = torch.zeros(2 * q.n_indenter_subdivisions, dtype=torch.float64, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    for _ in range(2):
        rc = f(C.byref(q), pts.data_ptr(), bins.data_ptr(), err.data_ptr(), n, None)
        assert rc == 0, im.library().icm_last_error()
    torch.cuda.synchronize()
    got = pts.cpu().numpy()

    e = compare_states(p, got, ref, soa)
    assert e["crushed_mismatch"] == 0 and e["grain_mismatch"] == 0
    assert max(e["disp_rel"], e["vel"], e["strain"], e["Bp"], e["Jp"]) < TOL, e
    assert max_rel(bins.cpu().numpy(), ref_bins) < TOL
    assert int(err.item()) == 0
    assert q.SimulationStep == ref_params.SimulationStep == 2 * n
    assert q.SimulationTime == ref_params.SimulationTime and q.indenter_x == ref_params.indenter_x


def test_noalloc_matches_the_oracle_on_the_70k_workload():
    """69,632 particles on the 512x128 grid (65,536 nodes, inside the
    scratch), 20 substeps in two calls, against the CPU oracle at the FP64
    tolerance of the other parity tests (the GPU's atomics reorder sums)."""
    import torch

    from icempm_b200 import configs
    from tests.mpm_cases import oracle_run

    p, soa = configs.make_scene("c1_70k")
    n = 10
    q_ref, ref, ref_bins, err_ref, _ = oracle_run(p, soa, 2 * n, threads=8)
    f = _noalloc()
    q = p.copy()
    pts = torch.tensor(soa, dtype=torch.float64, device="cuda")
    bins = torch.zeros(2 * q.n_indenter_subdivisions, dtype=torch.float64, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    for _ in range(2):
        rc = f(C.byref(q), pts.data_ptr(), bins.data_ptr(), err.data_ptr(), n, None)
        assert rc == 0, im.library().icm_last_error()
    torch.cuda.synchronize()
    e = compare_states(p, pts.cpu().numpy(), ref, soa)
    assert e["crushed_mismatch"] == 0 and e["grain_mismatch"] == 0
    assert max(e["disp_rel"], e["vel"], e["strain"], e["Bp"], e["Jp"]) < TOL, e
    assert np.abs(ref_bins).max() > 0 and max_rel(bins.cpu().numpy(), ref_bins) < TOL
    assert int(err.item()) == err_ref == 0
    assert q.SimulationStep == q_ref.SimulationStep and q.indenter_x == q_ref.indenter_x


def test_noalloc_rejects_grids_beyond_its_scratch():
    import torch

    p = params(1024, 257, dim=4.0, dt=1e-6)
    pts = torch.zeros(16 * 64, dtype=torch.float64, device="cuda")
    bins = torch.zeros(2 * p.n_indenter_subdivisions, dtype=torch.float64, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    p.nPts = 0
    p.nPtsPitch = 64
    rc = _noalloc()(C.byref(p), pts.data_ptr(), bins.data_ptr(), err.data_ptr(), 1, None)
    assert rc == 2
    assert b"exceeds the fixed grid scratch" in im.library().icm_last_error()
