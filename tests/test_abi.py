"""The C ABI library: loads without a GPU, exports every entry point that
include/*.h declares, and reports failures as status codes."""
import ctypes as C
import os
import re

import pytest

import icempm_b200 as im

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if not f.endswith(".h"):
            continue
        text = open(os.path.join(ROOT, "include", f)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(icm_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_every_declared_symbol_is_exported():
    names = declared_symbols()
    assert len(names) >= 30
    L = C.CDLL(im.LIB_PATH)
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing


def test_version_and_pitch():
    L = im.library()
    assert b"sm_100a" in L.icm_version()
    assert im.pitch_elems(1) == 64 and im.pitch_elems(64) == 64 and im.pitch_elems(65) == 128


def test_null_arguments_are_errors_not_crashes():
    L = im.library()
    assert L.icm_run_substeps(None, None, 1) == 2
    assert b"null" in L.icm_last_error()
    assert L.icm_transfer_points_to_device(None, None) == 2
    assert L.icm_scene_block(None, None, None, None) == 2
    assert L.icm_set_tile_split(None, 64, 1.3) == 2
    from icempm_b200 import ensemble as ens

    E = ens._sigs()
    assert E.icm_ensemble_set_split(None, 64, 1.3) == 2
    assert E.icm_ensemble_set(None, 200, 1) == 2
    assert E.icm_ensemble_run(None, None, 1) == 2
    assert E.icm_ensemble_size(None) == -1


@pytest.mark.skipif(os.path.exists("/dev/nvidia0"), reason="checks the no-device error path")
def test_create_without_device_reports_no_device():
    ctx = C.c_void_p()
    rc = im.library().icm_create(C.byref(ctx), 0)
    assert rc == 7
    g = im.GPU_Implementation5()
    with pytest.raises(RuntimeError, match="CUDA"):
        g.initialize()
