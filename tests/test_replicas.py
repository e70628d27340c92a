"""Multi-GPU is replicas only: every rank runs the whole workload on its own
GPU, the job time is the slowest rank's and the job rate counts all ranks'
particle-updates. These tests run the host side of that with the gloo
backend on CPU (world size 2) and the reference arm's rank handling."""
import json
import os
import socket
import subprocess
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _replica(rank, world, port, out):
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        # rank r's timed region took 1.5 + r seconds for 1000 units
        t = bench.max_over_ranks(1.5 + rank, dist, "cpu")
        out[rank] = (t, bench.job_rate(world, 1000, t))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_and_job_rate_gloo():
    world = 2
    with mp.get_context("spawn").Manager() as mgr:
        out = mgr.dict()
        mp.start_processes(_replica, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
        res = dict(out)
    for r in range(world):
        t, rate = res[r]
        assert t == 2.5  # the slowest rank's time on every rank
        assert rate == world * 1000 / 2.5


def test_single_process_helpers():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.max_over_ranks(3.0) == 3.0
    assert bench.job_rate(1, 100, 2.0) == 50.0


def _run_bench(env_extra, *args):
    env = dict(os.environ, **env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), *args], capture_output=True, text=True,
                          env=env, timeout=600)


def test_reference_arm_nonzero_rank_exits_quietly():
    r = _run_bench({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}, "--impl", "reference", "--gpus", "2",
                   "--steps", "1", "--warmup", "0", "--config", "c1_70k")
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""


def test_reference_arm_rank0_prints_one_line():
    r = _run_bench({"RANK": "0", "WORLD_SIZE": "1", "LOCAL_RANK": "0"}, "--impl", "reference", "--steps", "1",
                   "--warmup", "0", "--config", "c1_70k")
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["unit"] == "particle-updates/s" and d["value"] > 0
    assert d["cpu_baseline"]["kind"] == "port" and d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"]["h2d_bytes_per_step"] == 0 and d["e2e"]["d2h_bytes_per_step"] == 0


@pytest.mark.gpu
def test_bench_line_carries_the_contract_keys():
    """One short bench run on the GPU prints one JSON line with every key the
    measurement contract names (the sections that take minutes are off)."""
    r = _run_bench({"RANK": "0", "WORLD_SIZE": "1", "LOCAL_RANK": "0"}, "--steps", "1", "--warmup", "3",
                   "--substeps", "10", "--config", "c1_70k", "--tile", "1", "--no-accuracy", "--no-fp64",
                   "--no-ensemble", "--no-cpu")
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "gpu_launches", "roofline", "clocks", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["value"] > 0 and d["n_gpus"] == 1 and d["gpu_launches"] == 1 * (10 + 2)
    for k in ("bound", "achieved", "peak", "unit", "frac", "traffic"):
        assert k in d["roofline"], k
    for k in ("value", "unit", "h2d_bytes_per_step", "d2h_bytes_per_step"):
        assert k in d["e2e"], k
    assert d["e2e"]["h2d_bytes_per_step"] > 0 and d["e2e"]["d2h_bytes_per_step"] > 0
    for k in ("sm_mhz", "sm_max_mhz", "reasons"):
        assert k in d["clocks"], k
    assert "workload" in d["config"]
