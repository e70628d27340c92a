"""Synthetic block scene (stand-in for SnapshotManager::LoadRawPoints,
simulation/snapshotmanager.cpp:186-304)."""
import numpy as np

import icempm_b200 as im
from tests.mpm_cases import params


def test_block_counts_volume_and_placement():
    p = params(512, 128, 4.0, 2e-6)
    soa = im.make_block(p, 256, 68, ind_y_above_floor=0.2, seed=12345)
    n = 4 * 256 * 68
    assert p.nPts == n == 69632
    h = p.cellsize
    assert p.ParticleVolume == p.Volume / n
    assert abs(p.ParticleVolume - h * h / 4) < 1e-12
    assert p.ParticleMass == p.ParticleVolume * p.Density
    pitch = im.pitch_elems(n)
    S = im.SoA(soa, pitch, n)
    # centred in x, lifted by 2h (snapshotmanager.cpp:244-250)
    assert abs((S.pos[0].min() + S.pos[0].max()) / 2 - 2.0) < h
    assert abs(S.pos[1].min() - (2 * h + p.ymin)) < 1e-6
    # indenter just touching the left face, 0.2 m above the block bottom
    assert abs(p.indenter_x - (S.pos[0].min() - 0.15)) < 1e-6
    assert abs(p.indenter_y - (S.pos[1].min() + 0.2)) < 1e-6
    assert np.all(S.Fe[0] == 1) and np.all(S.Fe[3] == 1) and np.all(S.Fe[1] == 0)
    assert np.all(S.Jp_inv == 1) and np.all(S.crushed == 0)
    assert S.grain.min() >= 0 and S.grain.max() > 100
    # positions are float32 values (Points_Raw_2D is read as float)
    assert np.all(S.pos.astype(np.float32).astype(np.float64) == S.pos)


def test_block_sorted_by_cell_and_deterministic():
    p = params(96, 48, 0.75)
    a = im.make_block(p, 40, 10, seed=3)
    b = im.make_block(p, 40, 10, seed=3)
    c = im.make_block(p, 40, 10, seed=4)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    n = p.nPts
    S = im.SoA(a, im.pitch_elems(n), n)
    # SortPoints key on the raw (unshifted, float) coordinates
    raw_x = (S.pos[0] - (S.pos[0] - p.xmin).min()).astype(np.float32)
    key = (((S.pos[1] - 2 * p.cellsize).astype(np.float32) * p.cellsize_inv - 0.5).astype(int) * p.GridX)
    assert np.all(np.diff(key) >= 0)
    assert raw_x.size == n
