"""The command-line driver (icempm_b200/cli/cm.cpp), the counterpart of the
reference's cli/main.cpp: simulation thread, per-frame snapshot thread,
console commands, snapshots and P/Q dumps, resume from a snapshot."""
import json
import os
import subprocess

import numpy as np
import pytest

from icempm_b200 import build

from h5_check import H5
from mpm_cases import MATERIAL


@pytest.fixture(scope="module")
def cm():
    path = build.build_cli()
    assert path and os.path.exists(path)
    return path


def _config(tmp_path, **over):
    cfg = dict(MATERIAL, GridX=96, GridY=48, GridXDimension=0.75, InitialTimeStep=2e-6)
    cfg.update(over)
    path = tmp_path / "config.json"
    path.write_text(json.dumps(cfg))
    return str(path)


def _run(cm, *args, stdin=subprocess.DEVNULL, timeout=300):
    return subprocess.run([cm, *args], capture_output=True, text=True, stdin=stdin, timeout=timeout)


def test_usage(cm):
    r = _run(cm)
    assert r.returncode == 2 and "usage: cm config.json" in r.stderr
    r = _run(cm, "c.json", "--form", "fp16")
    assert r.returncode == 2


def test_missing_config(cm, tmp_path):
    r = _run(cm, str(tmp_path / "none.json"), "--block", "8", "8", "--frames", "1")
    assert r.returncode == 1
    assert r.stderr.startswith("cm: ")


def test_no_device_or_one_frame(cm, tmp_path):
    r = _run(cm, _config(tmp_path), "--block", "24", "8", "--frames", "1", "--out", str(tmp_path / "o"), "--quiet")
    if r.returncode != 0:  # no CUDA device here: initialize() throws
        assert r.returncode == 1 and "No avaialble CUDA devices" in r.stderr
    else:
        assert "cm done: 1 frames" in r.stdout


@pytest.mark.gpu
def test_frames_snapshots_pq_and_resume(cm, tmp_path):
    cfg = _config(tmp_path)
    out = tmp_path / "run"
    r = _run(cm, cfg, "--block", "24", "8", "--frames", "2", "--form", "fp64", "--pq", "--out", str(out))
    assert r.returncode == 0, r.stdout + r.stderr
    assert "cm done: 2 frames, step 5000, error 0" in r.stdout
    for f in ("snapshots/d00001.h5", "snapshots/d00002.h5", "pq/pq00001.h5", "pq/pq00002.h5"):
        assert (out / f).exists(), f
    f1, f2 = H5(str(out / "snapshots/d00001.h5")), H5(str(out / "snapshots/d00002.h5"))
    a1, a2 = f1.attrs("Params"), f2.attrs("Params")
    assert a1["SimulationTime"][0] < a2["SimulationTime"][0] and a2["indenter_x"][0] > a1["indenter_x"][0]

    # resume from frame 1 and run one frame: frame 2 again
    out2 = tmp_path / "resumed"
    r = _run(cm, cfg, "--resume", str(out / "snapshots/d00001.h5"), "--frames", "1", "--form", "fp64",
             "--out", str(out2))
    assert r.returncode == 0, r.stdout + r.stderr
    assert "resumed from" in r.stdout and "step 5000" in r.stdout
    g2 = H5(str(out2 / "snapshots/d00002.h5"))
    b2 = g2.attrs("Params")
    for k in ("SimulationTime", "indenter_x", "nPts", "nPtsPitch"):
        assert b2[k][0] == a2[k][0], k
    n, pitch = int(a2["nPts"][0]), int(a2["nPtsPitch"][0])
    h = float(a2["cellsize"][0])
    x_run = f2.dataset("Points").reshape(16, pitch)[4:6, :n]
    x_res = g2.dataset("Points").reshape(16, pitch)[4:6, :n]
    # FP64 float atomics reorder sums between the two runs
    assert np.abs(x_run - x_res).max() <= 1e-9 * h


@pytest.mark.gpu
def test_quit_command(cm, tmp_path):
    cfg = _config(tmp_path, SimulationEndTime=1.0)
    out = tmp_path / "q"
    p = subprocess.Popen([cm, cfg, "--block", "24", "8", "--out", str(out), "--quiet"], stdin=subprocess.PIPE,
                         stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True)
    try:
        o, e = p.communicate("q\n", timeout=300)
    finally:
        if p.poll() is None:
            p.kill()
    assert p.returncode == 0, o + e
    assert "requested to save the snapshot and terminate" in o
    assert "cm done:" in o
    assert any((out / "snapshots").iterdir())
