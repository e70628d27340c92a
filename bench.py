#!/usr/bin/env python
"""Throughput of the MLS-MPM substep on B200: particle-updates/s at 1M
particles (2048x512 grid, 999,424 particles, dt 5e-7), FP32 strain form and
FP64 forms, through the C ABI of libicempm.so.

One bench step = one icm_run_substeps call of --substeps substeps (default
100; the hot path over the whole particle set, back to back as inside a
frame). L2 is flushed (256 MB write) before every timed step. Timing: CUDA
events on the library's stream, max over ranks.

  python bench.py [--gpus N --steps K --warmup W]      our arm (FP32 headline)
  python bench.py --impl reference                      CPU oracle arm

Multi-GPU: replicas only (each rank runs the full workload on its own GPU;
the substep has no cross-GPU exchange), scaling "weak".
"""
from __future__ import annotations

import argparse
import ctypes
import gc
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "particle-updates/s at 1M pts: FP32/learned vs plain FP64, 1 B200, ≤1% force err"
UNIT = "particle-updates/s"
L2_FLUSH_BYTES = 256 << 20
# spread of the FP64 form itself: runs from an initial Fe perturbed by seeded
# N(0, a^2) noise at each amplitude a, SPREAD_SEEDS seeds each
SPREAD_AMPLITUDES, SPREAD_SEEDS = (1e-9, 1e-8, 3e-8), 5
# workloads whose full 10,000-substep frame is compared with the CPU oracle
ORACLE_WORKLOADS = ("c1_70k", "c2_250k")
LATE_SUBSTEPS = 200  # launches timed after a full frame (crushed particles present)
# learned projection: pairs harvested from the 250k-particle workload
HARVEST_CONFIG, HARVEST_EVERY, HARVEST_CAP = "c2_250k", 5, 4_000_000
# more pairs, from cases with other materials and indenters: the first 16
# cases of the ensemble workload, 3,000 substeps
HARVEST_ENS_CASES, HARVEST_ENS_SUBSTEPS, HARVEST_ENS_CAP = 16, 3000, 1_000_000
SUR_STEPS, SUR_TILES, SUR_TOL = 3000, 296, 0.02  # 296 tiles: two CTAs on each of 148 SMs
# re-binning interval of the ensemble and of its per-case arms
ENS_REBIN = 200


def parse():
    a = argparse.ArgumentParser()
    a.add_argument("--gpus", type=int, default=1)
    a.add_argument("--steps", type=int, default=10)
    a.add_argument("--warmup", type=int, default=3)
    a.add_argument("--impl", choices=["ours", "reference"], default="ours")
    a.add_argument("--config", default="c3_1m")
    a.add_argument("--substeps", type=int, default=100)
    a.add_argument("--tile", type=int, default=-1, help="tile variant (-1: autotuned)")
    a.add_argument("--threads", type=int, default=128)
    a.add_argument("--no-e2e", action="store_true")
    a.add_argument("--no-accuracy", action="store_true")
    a.add_argument("--no-oracle-accuracy", action="store_true",
                   help="skip the full-frame comparisons with the CPU oracle (70k and 250k workloads)")
    a.add_argument("--no-cpu", action="store_true")
    a.add_argument("--no-fp64", action="store_true")
    a.add_argument("--no-surrogate", action="store_true")
    a.add_argument("--no-ensemble", action="store_true")
    a.add_argument("--ensemble-substeps", type=int, default=1000)
    a.add_argument("--ensemble-cases", type=int, default=64)
    a.add_argument("--form", choices=["fp32", "fp64"], default="fp32",
                   help="fused form of the headline (fp64: for profiling the FP64 fused kernel)")
    return a.parse_args()


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(x: float, dist=None, device: str = "cuda") -> float:
    """The largest x over all ranks (the job's time is its slowest
    replica's); x itself without a process group."""
    if dist is None:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world: int, units_per_rank: float, seconds: float) -> float:
    """Whole-job throughput of `world` replicas that each processed
    units_per_rank units, timed by the slowest."""
    return world * units_per_rank / seconds


class Clocks:
    """Samples nvidia-smi every 200 ms while the timed region runs."""

    def __init__(self, index: int):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                          "-i", str(self.index), "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            if len(r) > 8:
                for k, nm in enumerate(names):
                    if r[5 + k].lower() == "active":
                        reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def traffic_summary():
    """Per-launch DRAM bytes of the fused kernel from the committed ncu summary."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def alg_bytes(form: str, n: int, na: int, ng: int) -> float:
    """Algorithmic bytes of one substep of the MLS-MPM step (the roofline's
    numerator), per particle and per node of the reference's three-kernel
    substep (gpu_implementation5.cu:148-379):
    FP64: P2G read 96 + G2P read 59 + G2P write 105 = 260 B per particle;
      grid reset 24 + mass read 8 per node, P2G write 24 + update r/w 32 +
      G2P gather 16 per active node -> 32 Ng + 72 Na.
    FP32 (same fields in float): 48 + 31 + 53 = 132 B per particle,
      16 Ng + 36 Na."""
    if form == "fp32":
        return 132.0 * n + 16.0 * ng + 36.0 * na
    return 260.0 * n + 32.0 * ng + 72.0 * na


def fused_min_bytes(form: str, n: int, na: int) -> float:
    """Bytes the fused one-launch substep must move at least (its own data
    layout): fp32 particle state read 36 B (fraction, cell and meta word in
    one 16-byte vector, H 16, Jp 4) + written 32 B, grid 48 B per active node
    (read 16, scatter 16, zero 16); fp64 read 60 B + written 48 B, grid 96 B
    per active node."""
    if form == "fp32":
        return 68.0 * n + 48.0 * na
    return 108.0 * n + 96.0 * na


def cpu_oracle_rate(name: str, budget_s: float, max_substeps: int, threads: int):
    """Particle-updates/s of the CPU FP64 oracle on the workload (a bounded
    sample: substeps until the time budget is spent)."""
    from oracle import oracle as orc

    p, soa = orc.workload(name)
    grid = orc.new_grid(p)
    bins = np.zeros(2 * p.n_indenter_subdivisions)
    orc.run_substeps(p, soa, grid, bins, 1, threads=threads, history=False)  # warm
    done, t0 = 0, time.perf_counter()
    while done < max_substeps:
        orc.run_substeps(p, soa, grid, bins, 1, threads=threads, history=False)
        done += 1
        if time.perf_counter() - t0 > budget_s and done >= 2:
            break
    dt = time.perf_counter() - t0
    return p.nPts * done / dt, done, dt, p.nPts


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference(args, rank, world):
    if rank != 0:
        return
    from oracle import oracle as orc

    threads = host_threads()
    # parameters and particles from the oracle's own restatement of the
    # workload set-up (bit-identical to the product's): this arm loads only
    # oracle/libmpm_oracle.so
    p, soa = orc.workload(args.config)
    grid = orc.new_grid(p)
    bins = np.zeros(2 * p.n_indenter_subdivisions)
    sub = args.substeps  # substeps per step, as the GPU arm's step
    for _ in range(args.warmup):
        orc.run_substeps(p, soa, grid, bins, sub, threads=threads, history=False)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        orc.run_substeps(p, soa, grid, bins, sub, threads=threads, history=False)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    value = p.nPts * sub * args.steps / total
    out = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{args.config}: 2D MLS-MPM ice indentation, {p.nPts} particles, "
                               f"{p.GridX}x{p.GridY} grid, dt {p.InitialTimeStep:g}",
                   "substeps_per_step": sub, "l2": "n/a (CPU)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{sub} substeps per step of the {p.nPts}-particle workload, "
                                   f"FP64 CPU restatement of gpu_implementation5.cu, OpenMP {threads} threads"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    rank, world, local = dist_env()
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

    import torch

    import icempm_b200 as im
    from icempm_b200 import configs

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    def barrier():
        if dist is not None:
            dist.barrier()

    def rank_max(x: float) -> float:
        return max_over_ranks(x, dist, "cuda")

    name = args.config
    p0, soa0 = configs.make_scene(name)
    n, ng = p0.nPts, p0.GridTotal
    na = configs.active_nodes(p0, soa0)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def make(form, tile, threads=None):
        m = im.Model(local)
        m.prms = configs.make_params(name)
        m.gpu.model = m
        gx, gy, dim, dt, cx, cy, _ = configs.CONFIGS[name]
        m.load_block(cx, cy, 0.2, 0.05, 12345)
        m.gpu.set_form(form)
        m.gpu.set_tile(tile, threads or args.threads)
        return m

    def timed(m, steps, warmup, substeps, ktime=False, clocks=None):
        g = m.gpu
        ext = torch.cuda.ExternalStream(g.stream_handle())
        for _ in range(warmup):
            g.run_substeps(m.prms, substeps)
        g.synchronize()
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(steps)]
        barrier()
        torch.cuda.synchronize()
        g.synchronize()
        ctx = clocks if clocks is not None else _Null()
        with ctx:
            for k in range(steps):
                with torch.cuda.stream(ext):
                    flush.zero_()
                evs[k][0].record(ext)
                g.run_substeps(m.prms, substeps)
                evs[k][1].record(ext)
            g.synchronize()
            torch.cuda.synchronize()
        barrier()
        ms = [a.elapsed_time(b) for a, b in evs]
        kt = (0.0, 0)
        if ktime:
            # per-launch durations of the fused kernel: further steps with an
            # event pair around every launch, after the timed region (the
            # pairs stand between consecutive launches and cost them their
            # programmatic overlap, so these steps are not the value's)
            g.kernel_timing(True)
            for _ in range(max(2, steps // 3)):
                with torch.cuda.stream(ext):
                    flush.zero_()
                g.run_substeps(m.prms, substeps)
            g.synchronize()
            kt = g.kernel_time()
            g.kernel_timing(False)
        return ms, kt

    hform = im.FORM_FP32 if args.form == "fp32" else im.FORM_FP64
    # --- tile choice (autotuner cache, else default)
    tile = args.tile
    tune_note = "fixed"
    if tile < 0:
        from icempm_b200 import autotune

        tile, threads, tune_note = autotune.choose(name, hform, local)
        args.threads = threads

    # --- headline: FP32 fused form (or the FP64 fused form with --form fp64)
    m = make(hform, tile)
    clocks = Clocks(local)
    ms, (kms, klaunch) = timed(m, args.steps, args.warmup, args.substeps, ktime=True, clocks=clocks)
    total_s = rank_max(sum(ms) / 1e3)
    value = job_rate(world, n * args.substeps * args.steps, total_s)
    m.gpu.close()

    hbm, peak_kind = peaks()
    # the fused kernel's time per launch inside the timed region: the step
    # time per substep (it also carries the run's P2G prologue, final
    # launch, tile sort and the L2 flush, so it is an upper bound)
    kavg_s = sum(ms) / len(ms) / args.substeps / 1e3
    kinst_s = (kms / klaunch / 1e3) if klaunch else float("nan")
    ab = alg_bytes(args.form, n, na, ng)
    fb = fused_min_bytes(args.form, n, na)
    achieved = ab / kavg_s / 1e9
    tr = traffic_summary().get(args.form)
    roof = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
            "traffic": tr, "kernel": f"k_tile_substep<Pol{args.form[2:]},16x16,kModeFull>" if tile == 1 else
            f"k_tile_substep<Pol{args.form[2:]},{im.TILE_VARIANTS[tile]},kModeFull>",
            "alg_bytes_per_launch": ab, "avg_launch_us": kavg_s * 1e6,
            "launch_timing": "timed-region step time per substep (CUDA events on the library's stream); "
                             "consecutive launches overlap (programmatic dependent launch)",
            "instrumented_launch_us": kinst_s * 1e6, "instrumented_launches": klaunch,
            "instrumented_frac": ab / kinst_s / 1e9 / hbm,
            "peak_kind": peak_kind,
            "fused_min_bytes_per_launch": fb, "frac_of_fused_min_bytes": fb / kavg_s / 1e9 / hbm}

    extra = {}
    # --- FP64 forms (the plain drop-in and the fused FP64 form)
    tile64, threads64 = tile, args.threads
    if not args.no_fp64:
        if args.tile < 0:
            from icempm_b200 import autotune

            tile64, threads64, _ = autotune.choose(name, im.FORM_FP64, local)
        k2 = max(2, args.steps // 3)
        for form, key in ((im.FORM_FP64, "fp64_fused"), (im.FORM_FP64_STEPWISE, "fp64_stepwise")):
            mm = make(form, tile64, threads64)
            ms2, (k2ms, k2n) = timed(mm, k2, 1, args.substeps, ktime=(form == im.FORM_FP64))
            t2 = rank_max(sum(ms2) / 1e3)
            v2 = job_rate(world, n * args.substeps * k2, t2)
            d = {"value": v2, "ms_per_step": sum(ms2) / k2, "steps": k2,
                 "tile": im.TILE_VARIANTS[tile64] if form == im.FORM_FP64 else None,
                 "threads": threads64 if form == im.FORM_FP64 else None}
            if k2n:
                per = sum(ms2) / k2 / args.substeps / 1e3
                a2 = alg_bytes("fp64", n, na, ng) / per / 1e9
                d["roofline"] = {"achieved": a2, "frac": a2 / hbm, "avg_launch_us": per * 1e6,
                                 "instrumented_launch_us": 1e3 * k2ms / k2n,
                                 "traffic": traffic_summary().get("fp64")}
            else:
                # step-wise: reset + three kernels per substep, from the step time
                a2 = alg_bytes("fp64", n, na, ng) * args.substeps / (sum(ms2) / k2 / 1e3) / 1e9
                d["roofline"] = {"achieved": a2, "frac": a2 / hbm, "from": "step time (4 launches per substep)"}
            extra[key] = d
            mm.gpu.close()
        mc = make(im.FORM_FP32_COMPENSATED, tile)
        msc, _ = timed(mc, k2, 1, args.substeps)
        extra["fp32_compensated"] = {"value": job_rate(world, n * args.substeps * k2, rank_max(sum(msc) / 1e3)),
                                     "ms_per_step": sum(msc) / k2, "steps": k2,
                                     "avg_launch_us": sum(msc) / k2 / args.substeps * 1e3}
        mc.gpu.close()
        extra["speedup_fp32_vs_fp64_stepwise"] = value / extra["fp64_stepwise"]["value"]
        extra["speedup_fp32_vs_fp64_fused"] = value / extra["fp64_fused"]["value"]

    # --- accuracy of the FP32 form over a full 10,000-substep frame
    if not args.no_accuracy and rank == 0:
        nsub = configs.CONFIGS[name][6]
        res = {}
        strays = {}
        late = {}

        def late_launch_us(mm):
            """Average fused launch after the frame: the crushed zone at the
            indenter is then fully developed."""
            mm.gpu.kernel_timing(True)
            mm.gpu.run_substeps(mm.prms, LATE_SUBSTEPS)
            kms2, kn2 = mm.gpu.kernel_time()
            mm.gpu.kernel_timing(False)
            return 1e3 * kms2 / max(kn2, 1)

        # the FP32 form's state against the FP64 fused form's after 1, 10 and
        # 100 substeps from the same initial state
        early, early_c = {}, {}
        pm = int(p0.nPtsPitch)
        pair = [make(im.FORM_FP64, tile64, threads64), make(im.FORM_FP32, tile),
                make(im.FORM_FP32_COMPENSATED, tile)]
        done = 0

        def state_err(a, b):
            dfe = np.abs(b.Fe - a.Fe).max(axis=0)
            strain = np.abs(a.Fe - np.array([1.0, 0.0, 0.0, 1.0])[:, None]).max()
            return {
                "x_max_err_h": float(np.abs(b.pos - a.pos).max() / p0.cellsize),
                "v_rel_err": float(np.abs(b.vel - a.vel).max() / max(np.abs(a.vel).max(), 1e-30)),
                "Fe_err_rel_to_max_strain": float(dfe.max() / max(strain, 1e-30)),
                "Fe_err_p99_rel_to_max_strain": float(np.percentile(dfe, 99) / max(strain, 1e-30)),
                "Jp_inv_max_abs_err": float(np.abs(b.Jp_inv - a.Jp_inv).max()),
            }
        for target in (1, 10, 100):
            bufs = []
            for mm in pair:
                mm.gpu.run_substeps(mm.prms, target - done)
                mm.gpu.cuda_transfer_from_device()
                mm.gpu.synchronize()
                bufs.append(im.SoA(mm.gpu.tmp_transfer_buffer.copy(), pm, n))
            done = target
            early[str(target)] = state_err(bufs[0], bufs[1])
            early_c[str(target)] = state_err(bufs[0], bufs[2])
        for mm in pair:
            mm.gpu.close()

        redo_frame = 0
        for form in (im.FORM_FP64, im.FORM_FP32, im.FORM_FP64_STEPWISE, im.FORM_FP32_COMPENSATED):
            f32_like = form in (im.FORM_FP32, im.FORM_FP32_COMPENSATED)
            mm = make(form, tile if f32_like else tile64, None if f32_like else threads64)
            mm.gpu.run_substeps(mm.prms, nsub)
            if form == im.FORM_FP32:
                redo_frame = mm.gpu.fp64_redo_count()
            if form != im.FORM_FP64_STEPWISE:
                strays[form] = mm.gpu.stray_count()
            hist = mm.gpu.force_history(nsub)
            mm.gpu.cuda_transfer_from_device()
            mm.gpu.synchronize()
            res[form] = (hist, mm.gpu.tmp_transfer_buffer.copy(), mm.gpu.error_code)
            if form not in (im.FORM_FP64_STEPWISE, im.FORM_FP32_COMPENSATED):
                late[im.FORM_NAMES[form]] = late_launch_us(mm)
            mm.gpu.close()
        h64, s64, e64 = res[im.FORM_FP64]
        h32, s32, e32 = res[im.FORM_FP32]
        hsw, ssw, esw = res[im.FORM_FP64_STEPWISE]
        hc, sc_, ec = res[im.FORM_FP32_COMPENSATED]
        f64 = np.hypot(h64[:, 0], h64[:, 1])
        f32 = np.hypot(h32[:, 0], h32[:, 1])
        fsw = np.hypot(hsw[:, 0], hsw[:, 1])
        win = 100  # substeps per window of the smoothed force history

        def smooth(f):
            return f[: len(f) // win * win].reshape(-1, win).mean(axis=1)
        pitch = int(p0.nPtsPitch)

        def pos(sbuf):
            return sbuf[4 * pitch: 6 * pitch].reshape(2, pitch)[:, :n]
        x64 = pos(s64)

        def frame_errors(f, x):
            """A frame's errors against the unperturbed FP64 fused frame."""
            dx = np.abs(x - x64).max(axis=0) / p0.cellsize
            return {"peak_force_rel_err": float(abs(f.max() - f64.max()) / max(f64.max(), 1e-30)),
                    "peak_force_rel_err_100substep_avg": float(abs(smooth(f).max() - smooth(f64).max()) /
                                                               max(smooth(f64).max(), 1e-30)),
                    "frame_impulse_rel_err": float(abs(f.sum() - f64.sum()) / max(abs(f64.sum()), 1e-30)),
                    "max_pos_err_h": float(dx.max()), "p99_pos_err_h": float(np.percentile(dx, 99))}

        # spread of the FP64 form itself under tiny perturbations of the
        # initial strain: the same frame from Fe + a N(0, 1) noise
        spread = {}
        for amp in SPREAD_AMPLITUDES:
            runs = []
            for seed in range(SPREAD_SEEDS):
                mm = make(im.FORM_FP64, tile64, threads64)
                S = mm.gpu.soa()
                S.Fe[:] += amp * np.random.default_rng(1000 + seed).standard_normal(S.Fe.shape)
                mm.gpu.transfer_ponts_to_device()
                mm.gpu.run_substeps(mm.prms, nsub)
                hp = mm.gpu.force_history(nsub)
                mm.gpu.cuda_transfer_from_device()
                mm.gpu.synchronize()
                runs.append(frame_errors(np.hypot(hp[:, 0], hp[:, 1]), pos(mm.gpu.tmp_transfer_buffer)))
                mm.gpu.close()
            spread[f"{amp:g}"] = {k: sorted(r[k] for r in runs) for k in runs[0]}
        e32f = frame_errors(f32, pos(s32))
        e32c = frame_errors(np.hypot(hc[:, 0], hc[:, 1]), pos(sc_))

        def rank_in_spread(err):
            """For each measure: the share of the perturbed FP64 runs (all
            amplitudes) whose error is at least this one's."""
            out = {}
            for k, v in err.items():
                allv = [x for a in spread.values() for x in a[k]]
                out[k] = float(np.mean([x >= v for x in allv])) if allv else None
            return out

        extra["accuracy"] = {
            "substeps": nsub,
            "against": "fp64 fused form on the GPU, which tracks the CPU FP64 oracle to ~1e-12 over 10,000 "
                       "substeps on the 70k and 250k workloads (oracle section) and over 200 substeps here",
            "fp32_state_err_after_substeps": early,
            "peak_force_fp64_N": float(f64.max()), "peak_force_fp32_N": float(f32.max()),
            "fp32": e32f,
            "fp32_share_of_fp64_spread_at_least_as_large": rank_in_spread(e32f),
            "force_history_rel_l2": float(np.linalg.norm(f32 - f64) / max(np.linalg.norm(f64), 1e-30)),
            "fp64_spread_under_initial_strain_noise": {
                "seeds": SPREAD_SEEDS, "errors_sorted_by_amplitude": spread,
                "what": "FP64 fused frames from Fe + a N(0,1) (seeded), against the unperturbed FP64 frame"},
            "fp64_vs_fp64_stepwise": frame_errors(fsw, pos(ssw)),
            "fp32_compensated": {
                "what": "FP32 form with compensated (Kahan) per-cell momentum sums",
                "state_err_after_substeps": early_c, "frame": e32c,
                "share_of_fp64_spread_at_least_as_large": rank_in_spread(e32c)},
            "error_flags": [int(e64), int(e32), int(esw), int(ec)],
            "late_frame_us_per_launch": late,
            "fp64_redo_per_substep": redo_frame / nsub,
            "stray_particle_substeps": {"fp64": strays.get(im.FORM_FP64), "fp32": strays.get(im.FORM_FP32)},
        }
        # full frames of the smaller workloads against the CPU FP64 oracle
        if not args.no_oracle_accuracy:
            from tests.tracking import track

            vs = {}
            for cname in ORACLE_WORKLOADS:
                pc, soac = configs.make_scene(cname)
                ns_c = configs.CONFIGS[cname][6]
                cps = (1, 10, 100, 1000, ns_c)
                t0 = time.perf_counter()
                r = track(pc, soac, (im.FORM_FP64_STEPWISE, im.FORM_FP64, im.FORM_FP32), cps, host_threads())
                r["particles"] = int(pc.nPts)
                r["substeps"] = ns_c
                r["seconds"] = time.perf_counter() - t0
                vs[cname] = r
            extra["accuracy"]["vs_cpu_oracle"] = vs

        # --- the learned projection: pairs harvested from the FP32 form on the
        # 250k-particle workload, trained on the tensor cores, then the
        # surrogate form on this workload
        if not args.no_surrogate:
            from icempm_b200 import surrogate as sg

            t0 = time.perf_counter()
            mh = configs.load_model(HARVEST_CONFIG, local)
            mh.gpu.set_form(im.FORM_FP32)
            mh.gpu.set_tile(1, 128)
            sg.set_harvest(mh.gpu, HARVEST_CAP, HARVEST_EVERY)
            mh.gpu.run_substeps(mh.prms, configs.CONFIGS[HARVEST_CONFIG][6])
            xh, yh = sg.harvest_pairs(mh.gpu, mh.prms, HARVEST_CAP)
            mh.gpu.close()
            from icempm_b200.ensemble import Ensemble

            he = Ensemble(im.FORM_FP32, 1, 128, device=local)
            hms = [configs.c4_model(c, local) for c in configs.c4_cases()[:HARVEST_ENS_CASES]]
            for hm in hms:
                sg.set_harvest(hm.gpu, HARVEST_ENS_CAP, HARVEST_EVERY)
                he.add(hm)
            he.run(HARVEST_ENS_SUBSTEPS)
            n_c2 = len(xh)
            parts = [sg.harvest_pairs(hm.gpu, hm.prms, HARVEST_ENS_CAP) for hm in hms]
            he.close()
            for hm in hms:
                hm.gpu.close()
            xh = np.concatenate([xh] + [a for a, _ in parts])
            yh = np.concatenate([yh] + [b for _, b in parts])
            t1 = time.perf_counter()
            net, loss = sg.fit(xh, yh, steps=SUR_STEPS, batch_tiles=SUR_TILES, lr=3e-3, seed=0, device=local)
            t2 = time.perf_counter()
            # throughput at the start of the frame, as the headline
            mt = make(im.FORM_FP32_SURROGATE, tile, 128)
            sg.set_surrogate(mt.gpu, net, SUR_TOL)
            k2 = max(2, args.steps // 3)
            ms3, (k3ms, k3n) = timed(mt, k2, 1, args.substeps, ktime=True)
            mt.gpu.close()
            # accuracy over the full frame, and the late-frame launch
            ms_ = make(im.FORM_FP32_SURROGATE, tile, 128)
            sg.set_surrogate(ms_.gpu, net, SUR_TOL)
            ms_.gpu.run_substeps(ms_.prms, nsub)
            hs = ms_.gpu.force_history(nsub)
            ms_.gpu.cuda_transfer_from_device()
            ms_.gpu.synchronize()
            ss = ms_.gpu.tmp_transfer_buffer.copy()
            acc_n, exact_n = sg.counts(ms_.gpu)
            late_s = late_launch_us(ms_)
            ms_.gpu.close()
            fs = np.hypot(hs[:, 0], hs[:, 1])
            xs = ss[4 * pitch: 6 * pitch].reshape(2, pitch)[:, :n]
            v3 = n * args.substeps * k2 / (sum(ms3) / 1e3)
            per3 = sum(ms3) / k2 / args.substeps / 1e3
            a3 = alg_bytes("fp32", n, na, ng) / per3 / 1e9
            extra["surrogate"] = {
                "value": v3, "unit": UNIT, "ms_per_step": sum(ms3) / k2, "steps": k2,
                "speedup_vs_fp64_stepwise": (v3 / extra["fp64_stepwise"]["value"]) if "fp64_stepwise" in extra else None,
                "roofline": {"achieved": a3, "frac": a3 / hbm, "avg_launch_us": per3 * 1e6,
                             "instrumented_launch_us": 1e3 * k3ms / max(k3n, 1)},
                "late_frame_us_per_launch": late_s,
                "training": {"pairs": int(len(xh)), "harvested_from": f"{HARVEST_CONFIG}, FP32 form, every "
                                                                       f"{HARVEST_EVERY} substeps of a 10,000-substep frame "
                                                                       f"({n_c2} pairs), and the first {HARVEST_ENS_CASES} "
                                                                       f"ensemble cases over {HARVEST_ENS_SUBSTEPS} substeps "
                                                                       f"({len(xh) - n_c2} pairs)",
                             "steps": SUR_STEPS, "batch": 128 * SUR_TILES, "first_loss": float(loss[:10].mean()),
                             "final_loss": float(loss[-100:].mean()), "harvest_s": t1 - t0, "train_s": t2 - t1},
                "tolerance": SUR_TOL,
                "network_projections_accepted": acc_n, "exact_projections": exact_n,
                "accuracy_vs_fp64": frame_errors(fs, xs),
                "share_of_fp64_spread_at_least_as_large": rank_in_spread(frame_errors(fs, xs)),
            }

    # --- the 64-case ensemble: every case as its own run_substeps (one after
    # another, and all at once on their own streams) against one ensemble
    # launch per substep over all cases' active tiles
    if not args.no_ensemble and rank == 0 and world == 1:
        extra["ensemble"] = ensemble_section(args, local, flush)

    # --- end to end: one frame through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        nsub = configs.CONFIGS[name][6]
        mm = make(im.FORM_FP32, tile)
        g = mm.gpu
        host = g.tmp_transfer_buffer.copy()
        bytes_soa = 8 * int(mm.prms.nPtsPitch) * 16
        d2h = bytes_soa + 8 * 2 * mm.prms.n_indenter_subdivisions + 4
        prms0 = type(mm.prms)()
        ctypes.memmove(ctypes.byref(prms0), ctypes.byref(mm.prms), ctypes.sizeof(prms0))
        times, sub_times = [], []
        ext = torch.cuda.ExternalStream(g.stream_handle())
        for k in range(1 + 2):
            # every frame starts from the same state: particles and SimParams
            # (time, step, indenter position)
            g.tmp_transfer_buffer[:] = host
            ctypes.memmove(ctypes.byref(mm.prms), ctypes.byref(prms0), ctypes.sizeof(prms0))
            barrier()
            g.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            g.record_start()
            g.transfer_ponts_to_device()
            a.record(ext)
            g.run_substeps(mm.prms, nsub)
            b.record(ext)
            g.cuda_transfer_from_device()
            g.record_stop()
            g.synchronize()
            if k > 0:
                times.append(g.elapsed_ms() / 1e3)
                sub_times.append(a.elapsed_time(b) / 1e3)
        te = rank_max(sum(times))
        ts = rank_max(sum(sub_times))
        e2e = {"value": job_rate(world, n * nsub * len(times), te), "unit": UNIT, "h2d_bytes_per_step": bytes_soa,
               "d2h_bytes_per_step": d2h, "substeps_per_step": nsub, "steps": len(times),
               "what": "Model-level frame: H2D of the reference SoA from pinned memory, 10,000 substeps, "
                       "D2H of SoA + force bins + error word",
               # the same frames without the copies: the whole frame's
               # substeps (early and late) with the state resident in HBM
               "frame_substeps_only": {"value": job_rate(world, n * nsub * len(sub_times), ts), "unit": UNIT,
                                       "us_per_substep": 1e6 * ts / (nsub * len(sub_times))}}
        mm.gpu.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        thr = host_threads()
        rate, done, secs, npts = cpu_oracle_rate(name, 10.0, 200, thr)
        cpu = {"value": rate, "unit": UNIT, "cores": thr, "kind": "port",
               "sample": f"{done} substeps ({secs:.1f} s) of the {npts}-particle workload, FP64 CPU restatement "
                         f"of gpu_implementation5.cu (oracle/mpm_oracle.c), OpenMP {thr} threads"}

    if rank == 0:
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sum(ms) / len(ms), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32" if args.form == "fp32" else "f64", "data": "synthetic",
            "config": {"workload": f"{name}: 2D MLS-MPM ice indentation, {n} particles, {p0.GridX}x{p0.GridY} grid "
                                   f"(h = 1/{round(1 / p0.cellsize)} m), dt {p0.InitialTimeStep:g}, "
                                   f"{'FP32 strain form' if args.form == 'fp32' else 'FP64 fused form'}",
                       "substeps_per_step": args.substeps, "tile": im.TILE_VARIANTS[tile], "threads": args.threads,
                       "tile_choice": tune_note, "active_nodes": na,
                       "l2": "flushed (256 MB write) before every timed step", "parallelism": f"replicas x{world}"},
            # per step: P2G prologue, substeps-1 full launches, the final
            # launch, and the tile-order sort
            "gpu_launches": args.steps * (args.substeps + 2),
            "roofline": roof,
            "clocks": clocks.summary(),
            "cpu_baseline": cpu,
            "e2e": e2e,
        }
        out.update(extra)
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def ensemble_section(args, device, flush):
    """The 64-case workload three ways, each arm on a fresh set of the same
    seeded cases (same initial states, same substeps): every case's own
    run_substeps one after another; all cases on their own streams at once;
    one ensemble. The ensemble then continues to the workload's full
    horizon (5,000 substeps)."""
    import torch

    import icempm_b200 as im
    from icempm_b200 import autotune, configs
    from icempm_b200.ensemble import Ensemble

    S = args.ensemble_substeps
    horizon = max(S, configs.C4["substeps"]) if args.ensemble_cases == configs.C4["cases"] else S
    cases = configs.c4_cases()[: args.ensemble_cases]
    form = im.FORM_FP32
    WARM = 3  # warm-up substeps of every arm (packing)

    def fresh():
        ms = [configs.c4_model(c, device) for c in cases]
        for m in ms:
            m.gpu.set_form(form)
            m.gpu.set_rebin_interval(ENS_REBIN)  # as the ensemble arm
        return ms

    def close(ms):
        # every release happens here, before the next arm's timed runs
        for m in ms:
            m.gpu.close()
        ms.clear()
        gc.collect()
        torch.cuda.synchronize()

    def ev():
        return torch.cuda.Event(enable_timing=True)

    def warm(ms):
        for m in ms:
            m.gpu.set_tile(tile, threads)
            m.gpu.run_substeps(m.prms, WARM)
        for m in ms:
            m.gpu.synchronize()
        torch.cuda.synchronize()

    t0 = time.perf_counter()
    models = fresh()
    npts = int(sum(m.prms.nPts for m in models))
    sizes = (min(m.prms.nPts for m in models), max(m.prms.nPts for m in models))
    t_setup = time.perf_counter() - t0
    tile, threads, note = autotune.choose_ensemble(models, form, f"c4_{len(cases)}", substeps=10)
    close(models)

    # every case alone, one after another (each timed on its own stream)
    models = fresh()
    warm(models)
    seq_ms = 0.0
    for m in models:
        st = torch.cuda.ExternalStream(m.gpu.stream_handle())
        with torch.cuda.stream(st):
            flush.zero_()
        a, b = ev(), ev()
        a.record(st)
        m.gpu.run_substeps(m.prms, S)
        b.record(st)
        b.synchronize()
        seq_ms += a.elapsed_time(b)
    close(models)

    # every case on its own stream, all enqueued before any finishes
    models = fresh()
    warm(models)
    flush.zero_()
    a, b = ev(), ev()
    a.record()
    for m in models:
        st = torch.cuda.ExternalStream(m.gpu.stream_handle())
        st.wait_event(a)
        m.gpu.run_substeps(m.prms, S)
    for m in models:
        e = ev()
        e.record(torch.cuda.ExternalStream(m.gpu.stream_handle()))
        torch.cuda.current_stream().wait_event(e)
    b.record()
    b.synchronize()
    conc_ms = a.elapsed_time(b)
    close(models)

    # the ensemble: runs of S substeps up to the horizon; the first run
    # covers the same substeps as the per-case arms
    models = fresh()
    ens = Ensemble(form, tile, threads, device=device)
    ens.set(rebin_interval=ENS_REBIN)
    for m in models:
        ens.add(m)
    st = torch.cuda.ExternalStream(ens.stream_handle())
    ens.run(WARM)
    ens.synchronize()
    torch.cuda.synchronize()
    runs = max(1, horizon // S)
    evs = [(ev(), ev()) for _ in range(runs)]
    for k in range(runs):
        with torch.cuda.stream(st):
            flush.zero_()
        evs[k][0].record(st)
        ens.run(S)
        evs[k][1].record(st)
    ens.synchronize()
    run_ms = [x.elapsed_time(y) for x, y in evs]
    ens_ms = run_ms[0]
    for m in models:
        m.gpu.cuda_transfer_from_device()
    for m in models:
        m.gpu.synchronize()
    errs = [int(m.gpu.error_code) for m in models]
    ens.close()
    close(models)
    return {
        "workload": f"{len(cases)} indentation cases (seeded blocks of {sizes[0]}-{sizes[1]} particles, {npts} in "
                    f"all; grid {configs.C4['grid'][0]}x{configs.C4['grid'][1]} each; materials and indenters "
                    "vary), FP32 form",
        "value": npts * runs * S / (sum(run_ms) / 1e3), "unit": UNIT, "substeps": runs * S,
        "ms_per_substep": sum(run_ms) / (runs * S),
        "ms_per_substep_by_run": [x / S for x in run_ms],
        "first_run": {"substeps": S, "ensemble_ms_per_substep": ens_ms / S,
                      "sequential_ms_per_substep": seq_ms / S, "concurrent_streams_ms_per_substep": conc_ms / S,
                      "speedup_vs_sequential": seq_ms / ens_ms, "speedup_vs_concurrent_streams": conc_ms / ens_ms},
        "tile": im.TILE_VARIANTS[tile], "threads": threads, "tile_choice": note,
        "timing": f"every arm: fresh copies of the same cases, {WARM} warm-up substeps (packing), then timed runs "
                  f"of {S} substeps (re-binned every {ENS_REBIN}), L2 flushed before each. Ensemble: {runs} runs, segments "
                  "replayed from CUDA graphs (the first captures inside the first run); per-case arms: the first "
                  "run, through run_substeps",
        "gpu_launches_per_substep": 1,
        "setup_s_per_copy": t_setup, "error_words": sorted(set(errs)),
    }


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *a):
        return False


if __name__ == "__main__":
    main()
