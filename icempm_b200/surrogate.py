"""The learned Drucker-Prager projection (csrc/mlp.cuh, csrc/mlp.cu): a
6 -> 64 -> 64 -> 3 GELU network trained and evaluated on the GPU's tensor
cores, standing in for Wolper_Drucker_Prager (gpu_implementation5.cu:48-94)
in principal space. See include/icempm.h for the parameter layout.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _check, _lib

N_IN, N_HID, N_OUT = 6, 64, 3
OFF_W1 = 0
OFF_B1 = OFF_W1 + N_HID * N_IN
OFF_W2 = OFF_B1 + N_HID
OFF_B2 = OFF_W2 + N_HID * N_HID
OFF_W3 = OFF_B2 + N_HID
OFF_B3 = OFF_W3 + N_OUT * N_HID
OFF_XMU = OFF_B3 + N_OUT
OFF_XSD = OFF_XMU + N_IN
OFF_YMU = OFF_XSD + N_IN
OFF_YSD = OFF_YMU + N_OUT
N_FLOATS = OFF_YSD + N_OUT


class TrainCfg(C.Structure):
    _fields_ = [("steps", C.c_int), ("batch_tiles", C.c_int), ("lr", C.c_float), ("seed", C.c_uint32)]


def _sigs():
    L = _lib()
    if getattr(L, "_mlp_sigs", False):
        return L
    vp, i, f = C.c_void_p, C.c_int, C.c_float
    for name, res, args in (
        ("icm_mlp_floats", i, []),
        ("icm_mlp_normalise", i, [vp, vp, vp, i]),
        ("icm_mlp_train", i, [i, vp, vp, i, C.POINTER(TrainCfg), vp, vp]),
        ("icm_mlp_gradient", i, [i, vp, vp, vp, i, vp, vp]),
        ("icm_mlp_infer", i, [i, vp, vp, i, vp, i]),
        ("icm_set_surrogate", i, [vp, vp, f]),
        ("icm_surrogate_counts", i, [vp, C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong)]),
        ("icm_set_harvest", i, [vp, i, i]),
        ("icm_harvest_pairs", i, [vp, vp, vp, vp, i, C.POINTER(i)]),
    ):
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    L._mlp_sigs = True
    assert L.icm_mlp_floats() == N_FLOATS
    return L


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


def views(net: np.ndarray) -> dict:
    """Named views of a parameter vector."""
    return {
        "W1": net[OFF_W1:OFF_B1].reshape(N_HID, N_IN), "b1": net[OFF_B1:OFF_W2],
        "W2": net[OFF_W2:OFF_B2].reshape(N_HID, N_HID), "b2": net[OFF_B2:OFF_W3],
        "W3": net[OFF_W3:OFF_B3].reshape(N_OUT, N_HID), "b3": net[OFF_B3:OFF_XMU],
        "x_mu": net[OFF_XMU:OFF_XSD], "x_sd": net[OFF_XSD:OFF_YMU],
        "y_mu": net[OFF_YMU:OFF_YSD], "y_sd": net[OFF_YSD:N_FLOATS],
    }


def init_net(seed: int = 0) -> np.ndarray:
    """Seeded He-style initial weights, zero biases, identity normalisation."""
    rng = np.random.default_rng(seed)
    net = np.zeros(N_FLOATS, dtype=np.float32)
    v = views(net)
    v["W1"][:] = rng.standard_normal((N_HID, N_IN)) * np.sqrt(2.0 / N_IN)
    v["W2"][:] = rng.standard_normal((N_HID, N_HID)) * np.sqrt(2.0 / N_HID)
    v["W3"][:] = rng.standard_normal((N_OUT, N_HID)) * np.sqrt(1.0 / N_HID)
    v["x_sd"][:] = 1.0
    v["y_sd"][:] = 1.0
    return net


def normalise(net: np.ndarray, x: np.ndarray, y: np.ndarray) -> None:
    """Sets net's normalisation from the samples (in place)."""
    x, y = _f32(x), _f32(y)
    _check(_sigs().icm_mlp_normalise(net.ctypes.data, x.ctypes.data, y.ctypes.data, len(x)))


def train(net: np.ndarray, x: np.ndarray, y: np.ndarray, steps: int = 2000, batch_tiles: int = 64, lr: float = 2e-3,
          seed: int = 1, device: int = 0) -> np.ndarray:
    """Trains net in place on the GPU; returns the loss of every step."""
    x, y = _f32(x), _f32(y)
    assert net.dtype == np.float32 and net.size == N_FLOATS
    loss = np.zeros(max(steps, 1), dtype=np.float32)
    cfg = TrainCfg(steps, batch_tiles, lr, seed)
    _check(_sigs().icm_mlp_train(device, x.ctypes.data, y.ctypes.data, len(x), C.byref(cfg), net.ctypes.data,
                                 loss.ctypes.data))
    return loss[:steps]


def gradient(net: np.ndarray, x: np.ndarray, y: np.ndarray, device: int = 0):
    """(gradient in the parameter layout, loss) of one pass over all samples."""
    x, y = _f32(x), _f32(y)
    net = _f32(net)
    g = np.zeros(N_FLOATS, dtype=np.float32)
    loss = np.zeros(1, dtype=np.float32)
    _check(_sigs().icm_mlp_gradient(device, net.ctypes.data, x.ctypes.data, y.ctypes.data, len(x), g.ctypes.data,
                                    loss.ctypes.data))
    return g, float(loss[0])


def infer(net: np.ndarray, x: np.ndarray, warp_form: bool = False, device: int = 0) -> np.ndarray:
    """Denormalised outputs for inputs x (n x 6): the tensor-core batch form
    or the warp form the substep kernel uses."""
    x = _f32(x)
    net = _f32(net)
    y = np.zeros((len(x), N_OUT), dtype=np.float32)
    _check(_sigs().icm_mlp_infer(device, net.ctypes.data, x.ctypes.data, len(x), y.ctypes.data,
                                 1 if warp_form else 0))
    return y


# ------------------------------------------------- the surrogate form

def set_surrogate(gpu, net, tolerance: float = 0.02) -> None:
    """Gives a GPU_Implementation5 the network of its surrogate form
    (FORM_FP32_SURROGATE); None removes it."""
    gpu.initialize()
    if net is None:
        _check(_sigs().icm_set_surrogate(gpu._ctx, None, C.c_float(0)))
        return
    net = _f32(net)
    _check(_sigs().icm_set_surrogate(gpu._ctx, net.ctypes.data, C.c_float(tolerance)))


def counts(gpu):
    """(network projections accepted, exact projections) since set_surrogate."""
    a, e = C.c_ulonglong(0), C.c_ulonglong(0)
    _check(_sigs().icm_surrogate_counts(gpu._ctx, C.byref(a), C.byref(e)))
    return int(a.value), int(e.value)


def set_harvest(gpu, capacity: int, every: int = 1) -> None:
    """Record crushed particles' trial states on every `every`-th substep
    of the fused FP32 forms (capacity 0: off)."""
    gpu.initialize()
    _check(_sigs().icm_set_harvest(gpu._ctx, capacity, every))


def harvest_pairs(gpu, prms, cap: int):
    """The recorded states labelled by the exact projection: (x n x 6, y n x 3)."""
    x = np.zeros((cap, N_IN), dtype=np.float32)
    y = np.zeros((cap, N_OUT), dtype=np.float32)
    n = C.c_int(0)
    _check(_sigs().icm_harvest_pairs(gpu._ctx, C.byref(prms), x.ctypes.data, y.ctypes.data, cap, C.byref(n)))
    return x[: n.value], y[: n.value]


def fit(x: np.ndarray, y: np.ndarray, steps: int = 3000, batch_tiles: int = 32, lr: float = 3e-3, seed: int = 0,
        device: int = 0):
    """A network trained on labelled pairs: normalisation from the data,
    seeded initial weights, Adam on the tensor cores. Returns (net, loss)."""
    net = init_net(seed)
    normalise(net, x, y)
    loss = train(net, x, y, steps=steps, batch_tiles=batch_tiles, lr=lr, seed=seed + 1, device=device)
    return net, loss
