"""Many indentation cases advanced together on one GPU (icm_ensemble_* in
include/icempm.h): one launch per substep over the active tiles of every
case, replayed from a captured CUDA graph between re-binnings."""
from __future__ import annotations

import ctypes as C
from typing import List

from . import FORM_FP32, Model, SimParams, _check, _lib


def _sigs():
    L = _lib()
    if getattr(L, "_ens_sigs", False):
        return L
    vp, i = C.c_void_p, C.c_int
    for name, res, args in (
        ("icm_ensemble_create", i, [C.POINTER(vp), i, i, i, i]),
        ("icm_ensemble_destroy", i, [vp]),
        ("icm_ensemble_add", i, [vp, vp]),
        ("icm_ensemble_size", i, [vp]),
        ("icm_ensemble_set", i, [vp, i, i]),
        ("icm_ensemble_set_split", i, [vp, i, C.c_double]),
        ("icm_ensemble_run", i, [vp, C.POINTER(C.POINTER(SimParams)), i]),
        ("icm_ensemble_stream", vp, [vp]),
    ):
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    L._ens_sigs = True
    return L


class Ensemble:
    """Cases are Models (their own blocks, materials, indenters and grids)
    set up as for a single run; run(n) advances every case n substeps,
    leaving each case's results in its Model as run_substeps would."""

    def __init__(self, form: int = FORM_FP32, tile: int = 1, threads: int = 128, device: int = 0):
        self._e = C.c_void_p(None)
        _check(_sigs().icm_ensemble_create(C.byref(self._e), device, form, tile, threads))
        self.models: List[Model] = []

    def add(self, model: Model) -> int:
        model.gpu.initialize()
        _check(_sigs().icm_ensemble_add(self._e, model.gpu._ctx))
        self.models.append(model)
        return len(self.models) - 1

    def set(self, rebin_interval: int = 200, graphs: bool = True) -> None:
        _check(_sigs().icm_ensemble_set(self._e, rebin_interval, 1 if graphs else 0))

    def set_split(self, max_tiles: int = 128, ratio: float = 1.3) -> None:
        """Heavy tiles run as two CTAs. An ensemble starts with this off;
        set_split() turns it on with the single-run defaults, max_tiles 0
        turns it off again."""
        _check(_sigs().icm_ensemble_set_split(self._e, max_tiles, ratio))

    def run(self, n: int) -> None:
        arr = (C.POINTER(SimParams) * len(self.models))(*[C.pointer(m.prms) for m in self.models])
        _check(_sigs().icm_ensemble_run(self._e, arr, n))

    def stream_handle(self) -> int:
        return int(_sigs().icm_ensemble_stream(self._e) or 0)

    def synchronize(self) -> None:
        for m in self.models:
            m.gpu.synchronize()

    def close(self) -> None:
        if self._e:
            _sigs().icm_ensemble_destroy(self._e)
            self._e = C.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
