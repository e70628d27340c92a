"""Shared scene set-up and comparison helpers for the tests."""
from __future__ import annotations

import json

import numpy as np

import icempm_b200 as im
from oracle import oracle as orc

# Material and indenter of the headline configurations: rho 980, E 1e9,
# nu 0.3, DP_phi 62, DP_threshold_p 1e3, strengths 100/10/4.5 MPa,
# GrainVariability 0.5, cylinder r = 0.15 m moving at 0.2 m/s.
MATERIAL = {
    "InputRawPoints": "synthetic",
    "YoungsModulus": 1.0e9, "PoissonsRatio": 0.3, "Density": 980, "Gravity": 9.81,
    "IceCompressiveStrength": 100e6, "IceTensileStrength": 10e6, "IceShearStrength": 4.5e6,
    "DP_phi": 62, "DP_threshold_p": 1e3, "GrainVariability": 0.5,
    "IndDiameter": 0.3, "IndVelocity": 0.2, "SimulationEndTime": 12,
}


def params(grid_x=96, grid_y=48, dim=0.75, dt=2e-6, **over) -> im.SimParams:
    p = im.SimParams()
    p.Reset()
    d = dict(MATERIAL, GridX=grid_x, GridY=grid_y, GridXDimension=dim, InitialTimeStep=dt)
    d.update(over)
    p.ParseString(json.dumps(d))
    return p


def scene(p: im.SimParams, cells=(48, 12), seed=7, ind_y=0.05, perturb=0.0, vel=0.0, crushed_frac=0.0,
          jp_spread=0.0, shift_x=0.0):
    """A block scene; optional seeded perturbations exercise every branch of
    the constitutive model (crushed particles, Jp_inv != 1, sheared Fe)."""
    soa = im.make_block(p, cells[0], cells[1], ind_y_above_floor=ind_y, grain_size=0.02, seed=seed)
    p.nPtsPitch = im.pitch_elems(p.nPts)
    p.nGridPitch = im.pitch_elems(p.GridTotal)
    S = im.SoA(soa, p.nPtsPitch, p.nPts)
    rng = np.random.default_rng(seed)
    n = p.nPts
    if shift_x:
        S.pos[0] += shift_x
    if perturb:
        S.Fe[:] += perturb * rng.standard_normal((4, n))
    if vel:
        S.vel[:] = vel * rng.standard_normal((2, n))
        S.Bp[:] = vel / p.cellsize * 0.1 * rng.standard_normal((4, n))
    if crushed_frac:
        S.crushed[:] = (rng.random(n) < crushed_frac).astype(np.uint8)
    if jp_spread:
        S.Jp_inv[:] = 1.0 + jp_spread * rng.standard_normal(n)
    return soa


def gpu_model(p: im.SimParams, soa: np.ndarray, form: int, tile: int = 1, threads: int = 256) -> im.Model:
    m = im.Model()
    m.prms = p.copy()
    m.gpu.model = m
    m.gpu.cuda_allocate_arrays(p.GridTotal, p.nPts)
    m.gpu.tmp_transfer_buffer[: soa.size] = soa
    m.gpu.transfer_ponts_to_device()
    m.Prepare()
    m.gpu.set_form(form)
    m.gpu.set_tile(tile, threads)
    return m


def gpu_state(m: im.Model) -> np.ndarray:
    m.gpu.cuda_transfer_from_device()
    m.gpu.synchronize()
    return m.gpu.tmp_transfer_buffer.copy()


def oracle_run(p: im.SimParams, soa: np.ndarray, n: int, threads: int = 1):
    q = p.copy()
    s = soa.copy()
    grid = orc.new_grid(q)
    bins = np.zeros(2 * q.n_indenter_subdivisions)
    err, hist = orc.run_substeps(q, s, grid, bins, n, threads=threads)
    return q, s, bins, err, hist


def max_rel(a, b, scale=None):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = np.abs(b).max() if scale is None else scale
    if s == 0:
        return float(np.abs(a - b).max())
    return float(np.abs(a - b).max() / s)


def compare_states(p, got, ref, x0):
    """Errors of got vs ref (both SoA buffers), each relative to the scale
    of the reference field; displacement relative to the cell size."""
    G = im.SoA(got, p.nPtsPitch, p.nPts)
    R = im.SoA(ref, p.nPtsPitch, p.nPts)
    X0 = im.SoA(x0, p.nPtsPitch, p.nPts)
    eye = np.array([1.0, 0.0, 0.0, 1.0])[:, None]
    return {
        "disp_h": float(np.abs(G.pos - R.pos).max() / p.cellsize),
        "disp_rel": max_rel(G.pos - X0.pos, R.pos - X0.pos),
        "vel": max_rel(G.vel, R.vel),
        "strain": max_rel(G.Fe - eye, R.Fe - eye),
        "Bp": max_rel(G.Bp, R.Bp),
        "Jp": max_rel(G.Jp_inv - 1.0, R.Jp_inv - 1.0) if np.abs(R.Jp_inv - 1).max() > 0 else
        float(np.abs(G.Jp_inv - R.Jp_inv).max()),
        "crushed_mismatch": int((G.crushed != R.crushed).sum()),
        "grain_mismatch": int((G.grain != R.grain).sum()),
    }
