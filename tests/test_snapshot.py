"""SnapshotManager (simulation/snapshotmanager.cpp): full snapshots, resume
from a snapshot, P/Q dumps and raw point clouds, on the library's own HDF5
writer and reader. Files are also read by tests/h5_check.py, an independent
parser that is itself checked on files written by the HDF5 library (the
reference's geometries_2d/*.h5, when that tree is present)."""
import os

import numpy as np
import pytest

import icempm_b200 as im
from icempm_b200 import configs
from oracle import oracle as orc

from h5_check import H5
from mpm_cases import gpu_model, gpu_state, params, scene

from conftest import reference_root

_REF = reference_root()
FIXTURES = [os.path.join(_REF, "geometries_2d", f) for f in ("2d_70k.h5", "2d_250k.h5")] if _REF else []
ATTRS = ["indenter_x", "indenter_y", "SimulationTime", "GridX", "GridY", "nPts", "nPtsPitch", "UpdateEveryNthStep",
         "n_indenter_subdivisions", "cellsize", "IndDiameter", "InitialTimeStep", "SetupType", "Volume"]


def _case():
    p = params()
    soa = scene(p, perturb=1e-3, vel=0.05, crushed_frac=0.3, jp_spread=0.01)
    S = im.SoA(soa, p.nPtsPitch, p.nPts)
    rng = np.random.default_rng(3)
    S.rows[1, : p.nPts] = rng.standard_normal(p.nPts)  # P
    S.rows[2, : p.nPts] = rng.standard_normal(p.nPts)  # Q
    bins = rng.standard_normal(2 * p.n_indenter_subdivisions)
    p.SimulationStep = 3 * p.UpdateEveryNthStep + 7
    return p, soa, bins


def test_snapshot_round_trip(tmp_path):
    p, soa, bins = _case()
    path = im.save_snapshot_host(p, soa, bins, str(tmp_path))
    assert path.endswith(os.path.join("snapshots", "d00003.h5"))
    q, soa2, bins2 = im.read_snapshot_host(path)
    assert bytes(q) == bytes(p)
    assert np.array_equal(soa2.view(np.uint8), soa.view(np.uint8))
    assert np.array_equal(bins2, bins)


def test_snapshot_layout_independent_parser(tmp_path):
    p, soa, bins = _case()
    path = im.save_snapshot_host(p, soa, bins, str(tmp_path))
    f = H5(path)
    assert sorted(f.entries) == ["Indenter_2D", "Params", "Points"]
    assert f.superblock["leaf_k"] == 4 and f.superblock["internal_k"] == 16
    ind, prm, pts = f.dataset("Indenter_2D"), f.dataset("Params"), f.dataset("Points")
    assert ind.dtype == np.float64 and ind.shape == (2 * p.n_indenter_subdivisions,)
    assert prm.dtype == np.uint8 and prm.shape == (432,) and prm.tobytes() == bytes(p)
    assert pts.dtype == np.float64 and pts.shape == (16 * p.nPtsPitch,)
    assert np.array_equal(pts.view(np.uint8), soa.view(np.uint8)) and np.array_equal(ind, bins)
    a = f.attrs("Params")
    assert list(a) == ATTRS
    for k in ATTRS:
        assert a[k].shape == (1,)
        assert a[k][0] == getattr(p, k), k
    assert a["nPtsPitch"].dtype == np.int64 and a["GridX"].dtype == np.int32 and a["Volume"].dtype == np.float64


def test_save_pq_splits_by_crushed(tmp_path):
    p, soa, bins = _case()
    path = im.save_pq_host(p, soa, str(tmp_path))
    assert path.endswith(os.path.join("pq", "pq00003.h5"))
    S = im.SoA(soa, p.nPtsPitch, p.nPts)
    f = H5(path)
    cr = f.dataset("PQ_crushed")
    it = f.dataset("PQ_intact")
    mask = S.crushed.astype(bool)
    assert cr.shape == (mask.sum(), 2) and it.shape == ((~mask).sum(), 2)
    assert np.array_equal(cr[:, 0], S.rows[1, : p.nPts][mask]) and np.array_equal(cr[:, 1], S.rows[2, : p.nPts][mask])
    assert np.array_equal(it[:, 0], S.rows[1, : p.nPts][~mask]) and np.array_equal(it[:, 1], S.rows[2, : p.nPts][~mask])
    assert list(f.attrs("PQ_intact")) == ATTRS and f.attrs("PQ_crushed") == {}


def test_save_pq_empty_set(tmp_path):
    p, soa, _ = _case()
    S = im.SoA(soa, p.nPtsPitch, p.nPts)
    S.crushed[:] = 0
    f = H5(im.save_pq_host(p, soa, str(tmp_path)))
    assert f.dataset("PQ_crushed").shape == (0, 2)
    assert f.dataset("PQ_intact").shape == (p.nPts, 2)


def test_read_snapshot_rejects_wrong_buffer(tmp_path):
    p, soa, bins = _case()
    path = im.save_snapshot_host(p, soa, bins, str(tmp_path))
    small = np.zeros(10)
    with pytest.raises(RuntimeError, match="Points size"):
        im._check(im.library().icm_read_snapshot(path.encode(), small.ctypes.data, small.size, None, 0))
    with pytest.raises(RuntimeError):
        im.read_snapshot_host(str(tmp_path / "missing.h5"))


def test_resume_is_exact_on_the_oracle(tmp_path):
    """A run interrupted by a snapshot and resumed from it continues exactly:
    the CPU oracle (deterministic) over 2 x 6 substeps against 12 straight."""
    p0 = params()
    soa0 = scene(p0, vel=0.05)
    p1, s1 = p0.copy(), soa0.copy()
    g1, b1 = orc.new_grid(p1), np.zeros(2 * p1.n_indenter_subdivisions)
    orc.run_substeps(p1, s1, g1, b1, 12, threads=1, history=False)

    p2, s2 = p0.copy(), soa0.copy()
    g2, b2 = orc.new_grid(p2), np.zeros(2 * p2.n_indenter_subdivisions)
    orc.run_substeps(p2, s2, g2, b2, 6, threads=1, history=False)
    path = im.save_snapshot_host(p2, s2, b2, str(tmp_path))
    p3, s3, b3 = im.read_snapshot_host(path)
    g3 = orc.new_grid(p3)
    orc.run_substeps(p3, s3, g3, b3, 6, threads=1, history=False)
    assert p3.SimulationStep == p1.SimulationStep and p3.SimulationTime == p1.SimulationTime
    assert np.array_equal(s3.view(np.uint8), s1.view(np.uint8))
    assert np.array_equal(b3, b1)


def test_repitch_soa_moves_grains_and_crushed():
    p, soa, _ = _case()
    n, pitch = p.nPts, p.nPtsPitch
    dst = np.zeros((pitch + 64) * 16)
    im.repitch_soa(soa, pitch, n, dst, pitch + 64)
    A, B = im.SoA(soa, pitch, n), im.SoA(dst, pitch + 64, n)
    assert np.array_equal(A.crushed, B.crushed) and np.array_equal(A.grain, B.grain)
    assert np.array_equal(A.rows[1:, :n], B.rows[1:, :n])


@pytest.mark.skipif(not FIXTURES or not os.path.exists(FIXTURES[0]), reason="reference fixtures not present")
@pytest.mark.parametrize("path", FIXTURES)
def test_raw_points_loader_matches_independent_parser(path):
    """LoadRawPoints on a file written by the HDF5 library (chunked,
    deflate): both readers agree; placement follows snapshotmanager.cpp:244-268."""
    if not os.path.exists(path):
        pytest.skip("fixture missing")
    f = H5(path)
    xy, gid = f.dataset("Points_Raw_2D"), f.dataset("GrainIDs")
    vol = float(f.attrs("GrainIDs")["volume"][0])
    p = configs.make_params("c2_250k")
    p.SortPointsByGridCell = 0
    soa = im.load_raw_points_host(p, path)
    n = len(gid)
    S = im.SoA(soa, p.nPtsPitch, n)
    assert p.nPts == n and p.Volume == vol
    assert np.array_equal(S.grain, gid)
    h = p.cellsize
    x_off = (p.GridX * h - float(np.float32(p.xmax - p.xmin))) / 2
    assert np.array_equal(S.pos[0], (xy[:, 0].astype(np.float64) + x_off).astype(np.float32))
    assert np.array_equal(S.pos[1], (xy[:, 1].astype(np.float64) + 2 * h).astype(np.float32))
    assert p.ParticleVolume == vol / n and p.ParticleMass == p.ParticleVolume * p.Density
    r = p.IndDiameter / 2
    ht = r - p.IndDepth
    assert p.indenter_x == np.floor((x_off - np.sqrt(r * r - ht * ht)) / h) * h
    assert p.indenter_y == p.ymax + 2 * h + ht
    # sorted load: same multiset of points, ordered by the SortPoints key
    q = configs.make_params("c2_250k")
    soa2 = im.load_raw_points_host(q, path)
    T = im.SoA(soa2, q.nPtsPitch, n)
    key = (((T.pos[0] - x_off).astype(np.float32) * q.cellsize_inv - 0.5).astype(np.int64)
           + (((T.pos[1] - 2 * h).astype(np.float32) * q.cellsize_inv - 0.5).astype(np.int64)) * q.GridX)
    assert np.all(np.diff(key) >= 0)
    assert np.array_equal(np.sort(T.grain), np.sort(gid))


def test_raw_points_errors(tmp_path):
    p = configs.make_params("c1_70k")
    with pytest.raises(RuntimeError, match="no file"):
        im.load_raw_points_host(p, str(tmp_path / "none.h5"))
    bad = tmp_path / "bad.h5"
    bad.write_bytes(b"not hdf5 at all" * 10)
    with pytest.raises(RuntimeError, match="not an HDF5 file"):
        im.load_raw_points_host(p, str(bad))
    # a snapshot is HDF5 but has no Points_Raw_2D
    q, soa, bins = _case()
    path = im.save_snapshot_host(q, soa, bins, str(tmp_path))
    with pytest.raises(RuntimeError, match="Points_Raw_2D"):
        im.load_raw_points_host(p, path)


@pytest.mark.gpu
@pytest.mark.parametrize("form", [im.FORM_FP64_STEPWISE, im.FORM_FP64, im.FORM_FP32])
def test_resume_on_gpu(tmp_path, form):
    """Frame 1, SaveSnapshot, frame 2 against ReadSnapshot into a fresh Model
    and frame 2 there."""
    p = params()
    soa = scene(p, vel=0.05)

    def frame(m):
        m.gpu.cuda_reset_indenter_force_accumulator()
        n = 20 - m.prms.SimulationStep % 20
        m.gpu.run_substeps(m.prms, n)
        return gpu_state(m)

    m1 = gpu_model(p, soa, form)
    m1.prms.UpdateEveryNthStep = 20
    frame(m1)
    m1.gpu.host_side_indenter_force_accumulator[:] = 0
    path = im.SnapshotManager(m1).SaveSnapshot(str(tmp_path))
    want = frame(m1)
    p_want = m1.prms.copy()
    m1.gpu.close()

    m2 = im.Model(0)
    m2.gpu.set_form(form)
    m2.gpu.set_tile(1, 256)
    frame_no = im.SnapshotManager(m2).ReadSnapshot(path)
    assert frame_no == 1 and m2.prms.SimulationStep == 20
    got = frame(m2)
    assert m2.prms.SimulationStep == p_want.SimulationStep
    assert m2.prms.SimulationTime == p_want.SimulationTime
    n, pitch = p.nPts, int(m2.prms.nPtsPitch)
    a = got.reshape(16, pitch)[:, :n]
    b = want.reshape(16, int(p_want.nPtsPitch))[:, :n]
    tol = 1e-5 if form == im.FORM_FP32 else 1e-9
    assert np.abs(a[4:6] - b[4:6]).max() <= tol * p.cellsize
    m2.gpu.close()
