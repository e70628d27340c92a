"""SimParams layout, Reset, ParseFile and the derived constants
(simulation/parameters_sim.h:19-90, simulation/parameters_sim.cpp:5-155)."""
import ctypes as C
import json
import math
import os

import pytest

import icempm_b200 as im

# offsets of icy::SimParams measured from the reference header with g++ (x86-64)
OFFSETS = {
    "grid_array": 0, "indenter_force_accumulator": 8, "pts_array": 16, "nPtsPitch": 24, "nGridPitch": 32,
    "n_indenter_subdivisions": 40, "tpb_P2G": 44, "nPts": 56, "GridX": 60, "GridXDimension": 72,
    "InitialTimeStep": 80, "Gravity": 96, "lambda_": 128, "IceCompressiveStrength": 152, "NACC_beta": 176,
    "DP_tan_phi": 200, "cellsize": 216, "UpdateEveryNthStep": 240, "IndDiameter": 248, "xmin": 280,
    "nxmin": 312, "ParticleVolume": 328, "SimulationStep": 352, "SimulationTime": 360, "indenter_x": 368,
    "Volume": 400, "SetupType": 408, "GrainVariability": 416, "UseWarpLevelReduction": 424,
    "SortPointsByGridCell": 428,
}


def test_layout_is_432_bytes_with_reference_offsets():
    assert C.sizeof(im.SimParams) == 432
    for name, off in OFFSETS.items():
        assert getattr(im.SimParams, name).offset == off, name


def test_reset_defaults():
    p = im.SimParams()
    p.Reset()
    assert p.n_indenter_subdivisions == 100
    assert p.InitialTimeStep == 3e-5 and p.GridX == 128 and p.GridY == 55
    assert p.tpb_P2G == 256 and p.tpb_Upd == 512 and p.tpb_G2P == 128
    assert p.SortPointsByGridCell == 1 and p.UseWarpLevelReduction == 0
    assert p.DP_tan_phi == pytest.approx(math.tan(30 * math.pi / 180), rel=1e-15)
    # derived (ComputeLame / ComputeCamClayParams2 / ComputeHelperVariables)
    E, nu = 5e8, 0.3
    lam = E * nu / ((1 + nu) * (1 - 2 * nu))
    mu = E / (2 * (1 + nu))
    assert p.lambda_ == lam and p.mu == mu and p.kappa == mu * 2.0 / 3.0 + lam
    assert p.cellsize == 3.33 / 128 and p.GridTotal == 128 * 55
    assert p.UpdateEveryNthStep == int(1.0 / (200 * 3e-5))
    beta = 1e6 / 100e6
    assert p.NACC_beta == beta
    assert p.NACC_M == pytest.approx((2 * 0.5e6 * math.sqrt(1 + 2 * beta)) / (100e6 * (1 + beta)), rel=1e-15)


@pytest.mark.parametrize("dt,expect", [(1e-5, 500), (2e-6, 2500), (1e-6, 5000), (5e-7, 10000), (3e-5, 166)])
def test_update_every_nth_step_truncates(dt, expect):
    p = im.SimParams()
    p.Reset()
    p.ParseString(json.dumps({"InputRawPoints": "x", "InitialTimeStep": dt}))
    assert p.UpdateEveryNthStep == expect


def test_parse_keys_and_raw_points(tmp_path):
    cfg = {"InputRawPoints": "geometries_2d/block.h5", "InitialTimeStep": 2e-6, "GridX": 512, "GridY": 128,
           "GridXDimension": 4.0, "YoungsModulus": 1e9, "PoissonsRatio": 0.3, "Gravity": 9.81, "Density": 980,
           "IndDiameter": 0.3, "IndVelocity": 0.2, "IndDepth": 0.1, "IceCompressiveStrength": 100e6,
           "IceTensileStrength": 10e6, "IceShearStrength": 4.5e6, "DP_phi": 62, "DP_threshold_p": 1e3,
           "GrainVariability": 0.5, "UseWarpLevelReduction": 1, "tpb_P2G": 128, "tpb_Upd": 256, "tpb_G2P": 64,
           "SortPointsByGridCell": 0, "ParticleViewSize": 4.1, "SimulationEndTime": 3}
    f = tmp_path / "cfg.json"
    f.write_text(json.dumps(cfg, indent=1))
    p = im.SimParams()
    p.Reset()
    assert p.ParseFile(str(f)) == "geometries_2d/block.h5"
    assert (p.GridX, p.GridY, p.tpb_P2G, p.tpb_Upd, p.tpb_G2P) == (512, 128, 128, 256, 64)
    assert p.SortPointsByGridCell == 0 and p.UseWarpLevelReduction == 1
    assert p.cellsize == 4.0 / 512 and p.cellsize_inv == 1 / (4.0 / 512)
    assert p.Dp_inv == 4.0 / (p.cellsize * p.cellsize)
    assert p.IndRSq == 0.3 * 0.3 / 4.0
    assert p.DP_tan_phi == math.tan(62 * math.pi / 180)
    assert p.UpdateEveryNthStep == 2500
    assert p.kappa == pytest.approx(1e9 / (3 * (1 - 2 * 0.3)), rel=1e-14)


def test_parse_errors(tmp_path):
    p = im.SimParams()
    p.Reset()
    with pytest.raises(RuntimeError, match="not found"):
        p.ParseFile(str(tmp_path / "missing.json"))
    with pytest.raises(RuntimeError, match="not JSON"):
        p.ParseString("{\"GridX\": 12,")
    with pytest.raises(RuntimeError, match="InputRawPoints"):
        p.ParseString(json.dumps({"GridX": 64}))
    with pytest.raises(RuntimeError, match="wrong type"):
        p.ParseString(json.dumps({"InputRawPoints": "x", "GridX": 1.5}))
    with pytest.raises(RuntimeError):
        p.ParseString(json.dumps({"InputRawPoints": "x", "GridX": 0}))


def test_bytes_roundtrip():
    p = im.SimParams()
    p.Reset()
    p.indenter_x = 1.25
    q = im.SimParams.from_bytes(p.to_bytes())
    assert q.to_bytes() == p.to_bytes()
