"""The synthetic indentation workloads the benchmarks and tests run.

Each is an ice block on the floor of a 4 m x 1 m domain at 4 particles per
cell (seeded jittered lattice, Voronoi grains of ~0.05 m), rho 980 kg/m^3,
E 1 GPa, nu 0.3, Drucker-Prager friction angle 62 deg, threshold pressure
1 kPa, compressive / tensile / shear strength 100 / 10 / 4.5 MPa, grain
variability 0.5, and a rigid cylinder of radius 0.15 m, centred 0.2 m above
the block bottom, starting just touching the block's left face and moving at
0.2 m/s in +x. No point-cloud file or public dataset is involved.
"""
from __future__ import annotations

import json

import numpy as np

from . import Model, SimParams, make_block, pitch_elems

MATERIAL = {
    "InputRawPoints": "synthetic",
    "YoungsModulus": 1.0e9, "PoissonsRatio": 0.3, "Density": 980, "Gravity": 9.81,
    "IceCompressiveStrength": 100e6, "IceTensileStrength": 10e6, "IceShearStrength": 4.5e6,
    "DP_phi": 62, "DP_threshold_p": 1e3, "GrainVariability": 0.5,
    "IndDiameter": 0.3, "IndVelocity": 0.2, "SimulationEndTime": 12,
}

# name: (GridX, GridY, GridXDimension, dt, block cells x, block cells y, substeps)
CONFIGS = {
    "c1_70k": (512, 128, 4.0, 2e-6, 256, 68, 10000),
    "c2_250k": (1024, 256, 4.0, 1e-6, 512, 122, 10000),
    "c3_1m": (2048, 512, 4.0, 5e-7, 1024, 244, 10000),
}


def make_params(name: str) -> SimParams:
    gx, gy, dim, dt, _, _, _ = CONFIGS[name]
    p = SimParams()
    p.Reset()
    p.ParseString(json.dumps(dict(MATERIAL, GridX=gx, GridY=gy, GridXDimension=dim, InitialTimeStep=dt)))
    return p


def make_scene(name: str, seed: int = 12345):
    """(params, particle SoA) of a workload; params carry host pitches."""
    p = make_params(name)
    _, _, _, _, cx, cy, _ = CONFIGS[name]
    soa = make_block(p, cx, cy, ind_y_above_floor=0.2, grain_size=0.05, seed=seed)
    p.nPtsPitch = pitch_elems(p.nPts)
    p.nGridPitch = pitch_elems(p.GridTotal)
    return p, soa


def load_model(name: str, device: int = 0, seed: int = 12345) -> Model:
    """A Model with the workload uploaded (LoadRawPoints-equivalent)."""
    gx, gy, dim, dt, cx, cy, _ = CONFIGS[name]
    m = Model(device)
    m.prms = make_params(name)
    m.gpu.model = m
    m.load_block(cx, cy, ind_y_above_floor=0.2, grain_size=0.05, seed=seed)
    return m


def active_nodes(p: SimParams, soa: np.ndarray) -> int:
    """Grid nodes reached by at least one particle stencil."""
    n = p.nPts
    pitch = int(p.nPtsPitch)
    x = soa[4 * pitch: 4 * pitch + n]
    y = soa[5 * pitch: 5 * pitch + n]
    bx = (x * p.cellsize_inv - 0.5).astype(np.int64)
    by = (y * p.cellsize_inv - 0.5).astype(np.int64)
    mark = np.zeros((p.GridY + 3, p.GridX + 3), dtype=bool)
    for i in range(3):
        for j in range(3):
            mark[np.clip(by + j, 0, p.GridY + 2), np.clip(bx + i, 0, p.GridX + 2)] = True
    return int(mark[: p.GridY, : p.GridX].sum())


# Ensemble of indentation cases: 64 cases on a 4 m x 1 m domain at
# h = 1/256 (1024 x 256 grid), dt 1e-6, 5,000 substeps. Per case: particle
# count log-uniform in [20k, 500k] (4 per cell), block aspect from a width
# U[0.5, 2.0] m and height U[0.2, 0.6] m (the block is then sized to the
# count), indenter speed U[0.05, 1.0] m/s, radius U[0.05, 0.2] m, friction
# angle U[45, 70] deg, Young's modulus U[5e8, 3e9] Pa.
C4 = dict(cases=64, grid=(1024, 256), dim=4.0, dt=1e-6, substeps=5000)


def c4_cases(cases: int = 64, seed: int = 12345, n_min: int = 20_000, n_max: int = 500_000):
    """Seeded case descriptions: (parameter overrides, cells_x, cells_y,
    indenter height above the block bottom)."""
    import numpy as np

    rng = np.random.default_rng(seed)
    gx, gy = C4["grid"]
    out = []
    for _ in range(cases):
        n = float(np.exp(rng.uniform(np.log(n_min), np.log(n_max))))
        w, hgt = rng.uniform(0.5, 2.0), rng.uniform(0.2, 0.6)
        cells = n / 4.0
        cy = max(8, int(round(np.sqrt(cells * hgt / w))))
        cx = int(round(cells / cy))
        # keep the block inside the domain with room for the indenter
        cx = min(cx, gx - 120)
        cy = min(cy, gy - 40)
        r = rng.uniform(0.05, 0.2)
        over = dict(IndVelocity=float(rng.uniform(0.05, 1.0)), IndDiameter=float(2 * r),
                    DP_phi=float(rng.uniform(45, 70)), YoungsModulus=float(rng.uniform(5e8, 3e9)))
        h = C4["dim"] / gx
        ind_y = min(0.5 * cy * h, r + 0.05)
        out.append((over, cx, cy, ind_y))
    return out


def c4_model(case, device: int = 0, seed: int = 12345) -> Model:
    """A Model holding one ensemble case (block loaded, constants set)."""
    over, cx, cy, ind_y = case
    gx, gy = C4["grid"]
    m = Model(device)
    p = SimParams()
    p.Reset()
    p.ParseString(json.dumps(dict(MATERIAL, GridX=gx, GridY=gy, GridXDimension=C4["dim"],
                                  InitialTimeStep=C4["dt"], **over)))
    m.prms = p
    m.gpu.model = m
    m.load_block(cx, cy, ind_y_above_floor=ind_y, grain_size=0.05, seed=seed)
    return m
