"""The autotuner's cache (icempm_b200/autotune.py): a cached choice is
returned without a sweep, keyed by GPU name, workload and form."""
import json

import icempm_b200 as im
from icempm_b200 import autotune


class _Gpu:
    _device = 0


class _Case:
    gpu = _Gpu()


def test_cached_ensemble_choice_skips_the_sweep(tmp_path, monkeypatch):
    cache = tmp_path / "tune.json"
    name = autotune._gpu_name(0)
    key = f"{name}|ensemble|c4_64|form{im.FORM_FP32}"
    cache.write_text(json.dumps({key: {"tile": 2, "threads": 128, "us": 460.0, "sweep": []}}))
    monkeypatch.setattr(autotune, "_CACHE", str(cache))

    def no_sweep(*a, **k):
        raise AssertionError("a cached choice must not sweep")

    monkeypatch.setattr(autotune, "sweep_ensemble", no_sweep)
    tile, threads, note = autotune.choose_ensemble([_Case()], im.FORM_FP32, "c4_64")
    assert (tile, threads) == (2, 128) and "cached" in note


def test_uncached_ensemble_choice_sweeps_and_stores(tmp_path, monkeypatch):
    cache = tmp_path / "tune.json"
    monkeypatch.setattr(autotune, "_CACHE", str(cache))
    calls = []

    def fake_sweep(models, form, substeps=20):
        calls.append(form)
        return [(0, 128, 900.0), (1, 128, 650.0), (3, 256, 700.0)]

    monkeypatch.setattr(autotune, "sweep_ensemble", fake_sweep)
    tile, threads, note = autotune.choose_ensemble([_Case()], im.FORM_FP64, "c4_8")
    assert (tile, threads) == (1, 128) and calls == [im.FORM_FP64]
    stored = json.loads(cache.read_text())
    (k, v), = stored.items()
    assert k.endswith(f"|ensemble|c4_8|form{im.FORM_FP64}") and v["tile"] == 1 and v["us"] == 650.0
    # the second call is served from the cache
    tile2, threads2, note2 = autotune.choose_ensemble([_Case()], im.FORM_FP64, "c4_8")
    assert (tile2, threads2) == (1, 128) and "cached" in note2 and len(calls) == 1
