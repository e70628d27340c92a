"""GPU runs against the CPU FP64 oracle over long horizons.

Both sides start from the same particle SoA and parameters and advance in
the same segments, so that their states can be compared at checkpoints
(after 1, 10, 100, ... substeps). Used by the parity tests at the
configurations the reference's step is quoted on, and by bench.py's
accuracy section. The oracle is the checker here, never the thing measured.
"""
from __future__ import annotations

import numpy as np

import icempm_b200 as im
from oracle import oracle as orc


def checkpoints_to_segments(checkpoints):
    out, done = [], 0
    for c in checkpoints:
        out.append(c - done)
        done = c
    return out


def oracle_track(p: im.SimParams, soa: np.ndarray, checkpoints, threads: int):
    """The oracle's states and per-substep force history at each checkpoint."""
    q = p.copy()
    s = soa.copy()
    grid = orc.new_grid(q)
    bins = np.zeros(2 * q.n_indenter_subdivisions)
    states, hist, err = [], [], 0
    for seg in checkpoints_to_segments(checkpoints):
        e, h = orc.run_substeps(q, s, grid, bins, seg, threads=threads)
        err |= e
        hist.append(h)
        states.append(s.copy())
    return states, np.concatenate(hist), bins, err


def gpu_track(p: im.SimParams, soa: np.ndarray, form: int, checkpoints, tile: int = 1, threads: int = 128,
              fp32_states=None):
    """The same on the GPU through the C ABI (Model + GPU_Implementation5);
    returns states, force history, bins, error word."""
    m = im.Model()
    m.prms = p.copy()
    m.gpu.model = m
    m.gpu.cuda_allocate_arrays(p.GridTotal, p.nPts)
    m.gpu.tmp_transfer_buffer[: soa.size] = soa
    m.gpu.transfer_ponts_to_device()
    m.Prepare()
    m.gpu.set_form(form)
    m.gpu.set_tile(tile, threads)
    m.gpu.cuda_reset_indenter_force_accumulator()
    states, hist = [], []
    try:
        for seg in checkpoints_to_segments(checkpoints):
            m.gpu.run_substeps(m.prms, seg)
            hist.append(m.gpu.force_history(seg))
            m.gpu.cuda_transfer_from_device()
            m.gpu.synchronize()
            states.append(m.gpu.tmp_transfer_buffer.copy())
        bins = m.gpu.host_side_indenter_force_accumulator.copy()
        err = m.gpu.error_code
    finally:
        m.gpu.close()
    return states, np.concatenate(hist), bins, err


def state_errors(p: im.SimParams, got: np.ndarray, ref: np.ndarray) -> dict:
    """Errors of a state against the oracle's: position in cells (max and
    99th percentile over particles), velocity relative to the largest
    velocity, Fe relative to the largest strain |Fe - I|, Jp_inv absolute,
    crushed flags that differ."""
    n, pitch = p.nPts, int(p.nPtsPitch)
    G = im.SoA(got, pitch, n)
    R = im.SoA(ref, pitch, n)
    eye = np.array([1.0, 0.0, 0.0, 1.0])[:, None]
    dx = np.abs(G.pos - R.pos).max(axis=0) / p.cellsize
    dfe = np.abs(G.Fe - R.Fe).max(axis=0)
    strain = max(float(np.abs(R.Fe - eye).max()), 1e-30)
    return {
        "x_max_h": float(dx.max()),
        "x_p99_h": float(np.percentile(dx, 99)),
        "v_rel": float(np.abs(G.vel - R.vel).max() / max(np.abs(R.vel).max(), 1e-30)),
        "Fe_rel": float(dfe.max() / strain),
        "Fe_p99_rel": float(np.percentile(dfe, 99) / strain),
        "Jp_inv_abs": float(np.abs(G.Jp_inv - R.Jp_inv).max()),
        "crushed_mismatch": int((G.crushed != R.crushed).sum()),
        "crushed": int(R.crushed.sum()),
    }


def force_errors(hist: np.ndarray, ref_hist: np.ndarray, window: int = 100) -> dict:
    """Indenter force history (per-substep summed reaction) against the
    oracle's: largest per-substep difference relative to the oracle's peak,
    the peaks' relative difference, and the same for the force averaged
    over windows of `window` substeps."""
    f = np.hypot(hist[:, 0], hist[:, 1])
    r = np.hypot(ref_hist[:, 0], ref_hist[:, 1])
    peak = max(float(r.max()), 1e-30)
    out = {"history_max_rel": float(np.abs(hist - ref_hist).max() / peak),
           "peak_rel": float(abs(f.max() - r.max()) / peak),
           "impulse_rel": float(abs(f.sum() - r.sum()) / max(float(r.sum()), 1e-30)),
           "peak_N": float(r.max())}
    if len(f) >= window:
        k = len(f) // window * window
        fs, rs = f[:k].reshape(-1, window).mean(axis=1), r[:k].reshape(-1, window).mean(axis=1)
        out["peak_rel_window_avg"] = float(abs(fs.max() - rs.max()) / max(float(rs.max()), 1e-30))
    return out


def track(p: im.SimParams, soa: np.ndarray, forms, checkpoints, threads: int, tile: int = 1, gpu_threads: int = 128):
    """Every form in `forms` against one oracle run: {form name:
    {checkpoint: state errors, "force": force errors, "error_word": ...}}."""
    ref_states, ref_hist, _, ref_err = oracle_track(p, soa, checkpoints, threads)
    out = {"oracle_error_word": int(ref_err)}
    for form in forms:
        states, hist, _, err = gpu_track(p, soa, form, checkpoints, tile, gpu_threads)
        r = {str(c): state_errors(p, s, rs) for c, s, rs in zip(checkpoints, states, ref_states)}
        r["force"] = force_errors(hist, ref_hist)
        r["error_word"] = int(err)
        out[im.FORM_NAMES[form]] = r
    return out
