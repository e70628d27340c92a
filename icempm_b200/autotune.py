"""Tile-shape / block-size autotuner for the fused substep kernel.

The reference fixes its launch shapes per kernel in SimParams (tpb_P2G,
tpb_Upd, tpb_G2P; simulation/parameters_sim.cpp:41-43). The fused kernel's
shape is a node tile (TX x TY, four built variants) and a block size; the
best pair depends on the particle count, the block geometry and the SM count.
``sweep`` times a short run of every pair with CUDA events on the library's
stream; ``choose`` returns the fastest and caches it per (GPU, particle
count, grid, form) in icempm_b200/_tune_cache.json.
"""
from __future__ import annotations

import json
import os
import threading

from . import TILE_VARIANTS

_CACHE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_tune_cache.json")
_LOCK = threading.Lock()
THREADS = (128, 256)


def sweep(model, substeps: int = 30, warmup: int = 5, variants=None, threads=THREADS):
    """[(variant, threads, microseconds per substep)] for every pair."""
    g = model.gpu
    out = []
    for v in (variants if variants is not None else sorted(TILE_VARIANTS)):
        for t in threads:
            g.set_tile(v, t)
            g.run_substeps(model.prms, warmup)
            g.synchronize()
            g.record_start()
            g.run_substeps(model.prms, substeps)
            g.record_stop()
            ms = g.elapsed_ms()
            out.append((v, t, 1e3 * ms / substeps))
    return out


def _key(gpu_name: str, model, form: int) -> str:
    p = model.prms
    return f"{gpu_name}|{p.nPts}|{p.GridX}x{p.GridY}|form{form}"


def _gpu_name(device: int) -> str:
    try:
        import torch

        return torch.cuda.get_device_name(device)
    except Exception:
        return "cuda"


def choose(config_name: str, form: int, device: int = 0, substeps: int = 30):
    """(tile variant, threads, note) for a workload of icempm_b200.configs."""
    from . import configs

    m = configs.load_model(config_name, device)
    m.gpu.set_form(form)
    key = _key(_gpu_name(device), m, form)
    with _LOCK:
        cache = {}
        if os.path.exists(_CACHE):
            try:
                with open(_CACHE) as f:
                    cache = json.load(f)
            except (OSError, ValueError):
                cache = {}
        if key in cache:
            c = cache[key]
            m.gpu.close()
            return c["tile"], c["threads"], f"autotuned (cached): {c['us']:.2f} us/substep"
    res = sweep(m, substeps=substeps)
    m.gpu.close()
    v, t, us = min(res, key=lambda x: x[2])
    with _LOCK:
        cache[key] = {"tile": v, "threads": t, "us": us, "sweep": res}
        try:
            with open(_CACHE, "w") as f:
                json.dump(cache, f, indent=1)
        except OSError:
            pass
    table = ", ".join(f"{TILE_VARIANTS[a][0]}x{TILE_VARIANTS[a][1]}/{b}: {c:.2f}" for a, b, c in res)
    return v, t, f"autotuned over {len(res)} shapes (us/substep: {table})"


def sweep_ensemble(models, form: int, substeps: int = 20, warmup: int = 4, variants=None, threads=THREADS,
                   rebin_interval: int = 200):
    """[(variant, threads, microseconds per substep of the whole ensemble)]:
    every pair timed on an ensemble of the given Models (their states
    advance during the sweep)."""
    import torch

    from .ensemble import Ensemble

    out = []
    for v in (variants if variants is not None else sorted(TILE_VARIANTS)):
        for t in threads:
            if TILE_VARIANTS[v][0] * TILE_VARIANTS[v][1] > 4 * t:
                continue
            ens = Ensemble(form, v, t, device=models[0].gpu._device)
            ens.set(rebin_interval=rebin_interval)
            for m in models:
                ens.add(m)
            ens.run(warmup)
            st = torch.cuda.ExternalStream(ens.stream_handle())
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ens.synchronize()
            a.record(st)
            ens.run(substeps)
            b.record(st)
            b.synchronize()
            out.append((v, t, 1e3 * a.elapsed_time(b) / substeps))
            ens.close()
    return out


def choose_ensemble(models, form: int, key: str, substeps: int = 20):
    """(tile variant, threads, note) for an ensemble, cached under key."""
    device = models[0].gpu._device
    full = f"{_gpu_name(device)}|ensemble|{key}|form{form}"
    with _LOCK:
        cache = {}
        if os.path.exists(_CACHE):
            try:
                with open(_CACHE) as f:
                    cache = json.load(f)
            except (OSError, ValueError):
                cache = {}
        if full in cache:
            c = cache[full]
            return c["tile"], c["threads"], f"autotuned (cached): {c['us']:.1f} us/substep"
    res = sweep_ensemble(models, form, substeps=substeps)
    v, t, us = min(res, key=lambda x: x[2])
    with _LOCK:
        cache[full] = {"tile": v, "threads": t, "us": us, "sweep": res}
        try:
            with open(_CACHE, "w") as f:
                json.dump(cache, f, indent=1)
        except OSError:
            pass
    table = ", ".join(f"{TILE_VARIANTS[a][0]}x{TILE_VARIANTS[a][1]}/{b}: {c:.1f}" for a, b, c in res)
    return v, t, f"autotuned over {len(res)} shapes (us/substep: {table})"
