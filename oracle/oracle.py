"""ctypes loader of the CPU FP64 oracle (oracle/mpm_oracle.c).

TEST INFRASTRUCTURE: imported only by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference legs, as the checker. The product path
never imports it.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libmpm_oracle.so")
REF_SVD_PATH = os.path.join(HERE, "_ref", "libref_svd.so")
REF_STEP_PATH = os.path.join(HERE, "_ref", "libref_step.so")

_L = None


def lib():
    global _L
    if _L is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} missing: run `make -C oracle`")
        from icempm_b200 import SimParams
        L = C.CDLL(LIB_PATH)
        P = C.POINTER(SimParams)
        vp, i, d = C.c_void_p, C.c_int, C.c_double
        sigs = {
            "oracle_svd2x2": (None, [vp, vp, vp, vp]),
            "oracle_kirchhoff": (None, [P, vp, vp]),
            "oracle_constitutive": (None, [P, vp, vp, vp, C.c_short, vp, vp]),
            "oracle_reset_grid": (None, [P, vp]),
            "oracle_p2g": (i, [P, vp, vp, i]),
            "oracle_update_nodes": (None, [P, vp, vp, d, d, vp, i]),
            "oracle_g2p": (None, [P, vp, vp, i, i]),
            "oracle_run_substeps": (i, [P, vp, vp, vp, vp, i, i]),
            "oracle_max_threads": (i, []),
            "oracle_compute_pq": (None, [P, vp, vp]),
            "oracle_grain_params": (None, [P, C.c_short, vp]),
            "oracle_failure_check": (i, [P, C.c_short, d, d]),
            "oracle_scene_block": (C.c_long, [P, i, i, d, d, C.c_uint64, vp]),
        }
        for n, (r, a) in sigs.items():
            f = getattr(L, n)
            f.restype = r
            f.argtypes = a
        _L = L
    return _L


def ref_svd_lib():
    """The reference's own SVD compiled for the host, or None if not built."""
    if not os.path.exists(REF_SVD_PATH):
        return None
    L = C.CDLL(REF_SVD_PATH)
    L.ref_svd.restype = None
    L.ref_svd.argtypes = [C.c_void_p] * 4
    return L


_RS = None


def ref_step_lib():
    """The reference's own device functions and kernel bodies
    (gpu_implementation5.cu:1-416) compiled for the host by
    oracle/build_ref.sh, or None if not built."""
    global _RS
    if _RS is None and os.path.exists(REF_STEP_PATH):
        L = C.CDLL(REF_STEP_PATH)
        vp, i, d = C.c_void_p, C.c_int, C.c_double
        sigs = {
            "ref_params_size": (i, []),
            "ref_kirchhoff": (None, [vp, vp, vp]),
            "ref_compute_pq": (None, [vp, vp, vp]),
            "ref_grain_params": (None, [vp, C.c_short, vp]),
            "ref_failure_check": (i, [vp, C.c_short, d, d]),
            "ref_constitutive": (None, [vp, vp, vp, vp, C.c_short, vp, vp]),
            "ref_run_substeps": (i, [vp, vp, vp, vp, i]),
        }
        for n, (r, a) in sigs.items():
            f = getattr(L, n)
            f.restype = r
            f.argtypes = a
        _RS = L
    return _RS


def compute_pq(prms, F):
    """ComputePQ: U[4], sigma[2], V[4], Je_tr, p_tr, q_tr, sigma^2[2],
    s_hat[2] as one array of 17."""
    F = np.ascontiguousarray(F, dtype=np.float64).reshape(4)
    out = np.zeros(17)
    lib().oracle_compute_pq(C.byref(prms), _p(F), _p(out))
    return out


def grain_params(prms, grain):
    out = np.zeros(5)
    lib().oracle_grain_params(C.byref(prms), int(grain), _p(out))
    return out


def failure_check(prms, grain, p, q) -> int:
    return int(lib().oracle_failure_check(C.byref(prms), int(grain), float(p), float(q)))


# ----------------------------------------------------------- parameters
# icy::SimParams set-up restated (simulation/parameters_sim.cpp): Reset
# (:5-56), the numeric keys of ParseFile (:73-98) and the derived constants
# (:121-147), in the reference's operation order, so that the CPU arm of
# bench.py builds its parameter block without the product library.

_DOUBLE_KEYS = ("InitialTimeStep", "YoungsModulus", "GridXDimension", "ParticleViewSize", "SimulationEndTime",
                "PoissonsRatio", "Gravity", "Density", "IndDiameter", "IndVelocity", "IndDepth",
                "IceCompressiveStrength", "IceTensileStrength", "IceShearStrength", "DP_threshold_p",
                "GrainVariability")
_INT_KEYS = ("GridX", "GridY", "UseWarpLevelReduction", "tpb_P2G", "tpb_Upd", "tpb_G2P", "SortPointsByGridCell")


def _derive(p):
    """ComputeCamClayParams2 (with ComputeLame) and ComputeHelperVariables."""
    E, nu = p.YoungsModulus, p.PoissonsRatio
    p.lambda_ = E * nu / ((1 + nu) * (1 - 2 * nu))
    p.mu = E / (2 * (1 + nu))
    p.kappa = p.mu * 2. / 3. + p.lambda_
    p.NACC_beta = p.IceTensileStrength / p.IceCompressiveStrength
    beta, q, p0 = p.NACC_beta, p.IceShearStrength, p.IceCompressiveStrength
    p.NACC_M = (2 * q * math.sqrt(1 + 2 * beta)) / (p0 * (1 + beta))
    p.NACC_Msq = p.NACC_M * p.NACC_M
    p.UpdateEveryNthStep = int(1.0 / (200 * p.InitialTimeStep))
    p.cellsize = p.GridXDimension / p.GridX
    p.cellsize_inv = 1. / p.cellsize
    p.Dp_inv = 4. / (p.cellsize * p.cellsize)
    p.IndRSq = p.IndDiameter * p.IndDiameter / 4.
    p.GridTotal = p.GridX * p.GridY


def params(values: dict):
    """A parameter block: Reset, then the configuration values (as ParseFile
    reads them; DP_phi in degrees), then the derived constants."""
    from icempm_b200 import SimParams  # the ctypes layout only

    p = SimParams()
    C.memset(C.byref(p), 0, C.sizeof(p))
    pi = 3.14159265358979323846
    p.n_indenter_subdivisions = 100
    p.InitialTimeStep = 3.e-5
    p.YoungsModulus = 5.e8
    p.GridX, p.GridY = 128, 55
    p.ParticleViewSize = 2.5
    p.GridXDimension = 3.33
    p.SimulationEndTime = 12
    p.PoissonsRatio, p.Gravity, p.Density = 0.3, 9.81, 980
    p.IndDiameter, p.IndVelocity, p.IndDepth = 0.324, 0.2, 0.25
    p.IceCompressiveStrength, p.IceTensileStrength, p.IceShearStrength = 100e6, 1e6, 0.5e6
    p.DP_tan_phi = math.tan(30 * pi / 180.)
    p.DP_threshold_p = 1e3
    p.tpb_P2G, p.tpb_Upd, p.tpb_G2P = 256, 512, 128
    p.GrainVariability = 0.50
    p.SortPointsByGridCell = 1
    _derive(p)
    for k in _DOUBLE_KEYS:
        if k in values:
            setattr(p, k, float(values[k]))
    for k in _INT_KEYS:
        if k in values:
            setattr(p, k, int(values[k]))
    if "DP_phi" in values:
        p.DP_tan_phi = math.tan(float(values["DP_phi"]) * pi / 180)
    _derive(p)
    return p


def scene_block(p, cells_x: int, cells_y: int, ind_y_above_floor: float, grain_size: float, seed: int):
    """The seeded synthetic block (oracle/scene_oracle.c); fills p and
    returns the particle SoA (16 rows of the 64-aligned pitch)."""
    n = 4 * cells_x * cells_y
    pitch = (n + 63) // 64 * 64
    soa = np.zeros(16 * pitch, dtype=np.float64)
    got = lib().oracle_scene_block(C.byref(p), cells_x, cells_y, ind_y_above_floor, grain_size, seed, _p(soa))
    if got != n:
        raise RuntimeError("oracle_scene_block failed")
    p.nPtsPitch = pitch
    p.nGridPitch = (p.GridTotal + 63) // 64 * 64
    return soa


def workload(name: str, seed: int = 12345):
    """(params, SoA) of a benchmark workload (icempm_b200.configs.CONFIGS),
    built by the oracle alone."""
    from icempm_b200 import configs  # the workload table (data only)

    gx, gy, dim, dt, cx, cy, _ = configs.CONFIGS[name]
    p = params(dict(configs.MATERIAL, GridX=gx, GridY=gy, GridXDimension=dim, InitialTimeStep=dt))
    return p, scene_block(p, cx, cy, 0.2, 0.05, seed)


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data


def svd2x2(A):
    """Row-major 2x2 -> (U row-major, sigma, V row-major) as the reference's
    svd2x2_modified returns them."""
    A = np.ascontiguousarray(A, dtype=np.float64).reshape(4)
    U, S, V = np.zeros(4), np.zeros(2), np.zeros(4)
    lib().oracle_svd2x2(_p(A), _p(U), _p(S), _p(V))
    return U, S, V


def constitutive(prms, Fe, Jp_inv, crushed, grain):
    Fe = np.ascontiguousarray(Fe, dtype=np.float64).reshape(4).copy()
    jp = np.array([Jp_inv], dtype=np.float64)
    cr = np.array([crushed], dtype=np.uint8)
    p = np.zeros(1)
    q = np.zeros(1)
    lib().oracle_constitutive(C.byref(prms), _p(Fe), _p(jp), cr.ctypes.data, int(grain), _p(p), _p(q))
    return Fe, float(jp[0]), int(cr[0]), float(p[0]), float(q[0])


def kirchhoff(prms, F):
    F = np.ascontiguousarray(F, dtype=np.float64).reshape(4)
    tau = np.zeros(4)
    lib().oracle_kirchhoff(C.byref(prms), _p(F), _p(tau))
    return tau


def new_grid(prms) -> np.ndarray:
    return np.zeros(int(prms.nGridPitch) * 3, dtype=np.float64)


def reset_grid(prms, grid):
    lib().oracle_reset_grid(C.byref(prms), _p(grid))


def p2g(prms, pts, grid, threads=1) -> int:
    return int(lib().oracle_p2g(C.byref(prms), _p(pts), _p(grid), threads))


def update_nodes(prms, grid, bins, ix, iy, threads=1):
    tot = np.zeros(2)
    lib().oracle_update_nodes(C.byref(prms), _p(grid), _p(bins), ix, iy, _p(tot), threads)
    return tot


def g2p(prms, pts, grid, record_pq, threads=1):
    lib().oracle_g2p(C.byref(prms), _p(pts), _p(grid), 1 if record_pq else 0, threads)


def run_substeps(prms, pts, grid, bins, n, threads=1, history=True):
    """Model::Step's substep loop on the CPU; returns (error, force history
    [n, 2] or None). Advances prms.SimulationStep / SimulationTime."""
    hist = np.zeros(2 * n) if history else None
    err = lib().oracle_run_substeps(C.byref(prms), _p(pts), _p(grid), _p(bins),
                                    _p(hist) if history else None, n, threads)
    return int(err), (hist.reshape(n, 2) if history else None)


def max_threads() -> int:
    return int(lib().oracle_max_threads())
