"""CPU oracle of the learned Drucker-Prager projection.

TEST INFRASTRUCTURE: imported only by tests/ as the checker of the GPU
network kernels (icempm_b200/csrc/mlp.cu) and of the training labels.

* dp_project: the exact projection in principal space, restated from
  Wolper_Drucker_Prager (gpu_implementation5.cu:48-94) with ComputePQ
  (:36-44); FP64.
* forward / backward: the 6 -> 64 -> 64 -> 3 tanh-GELU network in NumPy,
  with the operands of every product rounded to BF16 (round to nearest
  even) as the tensor-core kernels round them, FP32 everywhere else; the
  loss is the mean squared error over samples and the 3 outputs on
  normalised targets.
"""
from __future__ import annotations

import numpy as np

N_IN, N_HID, N_OUT = 6, 64, 3
SQRT2 = np.sqrt(2.0)


def _round(a: np.ndarray) -> np.ndarray:
    """Round-to-nearest-even to BF16, returned as float32."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def _gelu(z):
    c, a = np.float32(0.7978845608028654), np.float32(0.044715)
    return (np.float32(0.5) * z * (np.float32(1) + np.tanh(c * (z + a * z * z * z)))).astype(np.float32)


def _gelu_grad(z):
    c, a = np.float32(0.7978845608028654), np.float32(0.044715)
    th = np.tanh(c * (z + a * z * z * z))
    return (0.5 * (1 + th) + 0.5 * z * (1 - th * th) * c * (1 + 3 * a * z * z)).astype(np.float32)


def unpack(net: np.ndarray) -> dict:
    o = 0
    out = {}
    for name, shape in (("W1", (N_HID, N_IN)), ("b1", (N_HID,)), ("W2", (N_HID, N_HID)), ("b2", (N_HID,)),
                        ("W3", (N_OUT, N_HID)), ("b3", (N_OUT,)), ("x_mu", (N_IN,)), ("x_sd", (N_IN,)),
                        ("y_mu", (N_OUT,)), ("y_sd", (N_OUT,))):
        size = int(np.prod(shape))
        out[name] = np.asarray(net[o:o + size], dtype=np.float32).reshape(shape)
        o += size
    return out


def _ident(a):
    return np.asarray(a, dtype=np.float32)


def forward(net, x, keep=False, exact=False):
    """Normalised outputs for raw inputs x (n x 6); exact=True skips the
    BF16 rounding (for finite-difference checks)."""
    bf16 = _ident if exact else _round
    p = unpack(net)
    xn = bf16((np.asarray(x, np.float32) - p["x_mu"]) / p["x_sd"])
    z1 = (xn @ bf16(p["W1"]).T + p["b1"]).astype(np.float32)
    h1 = bf16(_gelu(z1))
    z2 = (h1 @ bf16(p["W2"]).T + p["b2"]).astype(np.float32)
    h2 = bf16(_gelu(z2))
    y = (h2 @ bf16(p["W3"]).T + p["b3"]).astype(np.float32)
    if keep:
        return y, (xn, z1, h1, z2, h2)
    return y


def predict(net, x):
    """Denormalised outputs."""
    p = unpack(net)
    return forward(net, x) * p["y_sd"] + p["y_mu"]


def backward(net, x, t, exact=False):
    """(gradient in the parameter layout, loss) over all samples."""
    bf16 = _ident if exact else _round
    p = unpack(net)
    n = len(x)
    y, (xn, z1, h1, z2, h2) = forward(net, x, keep=True, exact=exact)
    tn = ((np.asarray(t, np.float32) - p["y_mu"]) / p["y_sd"]).astype(np.float32)
    d = y - tn
    loss = float(np.sum(d.astype(np.float64) ** 2) / (3 * n))
    dy = (2.0 * d / (3 * n)).astype(np.float32)
    dz3 = bf16(dy)
    g = {}
    g["b3"] = dy.sum(0)
    g["W3"] = dz3.T @ h2
    dh2 = dz3 @ bf16(p["W3"])
    dz2 = (dh2 * _gelu_grad(z2)).astype(np.float32)
    g["b2"] = dz2.sum(0)
    dz2b = bf16(dz2)
    g["W2"] = dz2b.T @ h1
    dh1 = dz2b @ bf16(p["W2"])
    dz1 = (dh1 * _gelu_grad(z1)).astype(np.float32)
    g["b1"] = dz1.sum(0)
    g["W1"] = bf16(dz1).T @ xn[:, :N_IN]
    out = np.zeros_like(np.asarray(net, np.float32))
    o = 0
    for name, shape in (("W1", (N_HID, N_IN)), ("b1", (N_HID,)), ("W2", (N_HID, N_HID)), ("b2", (N_HID,)),
                        ("W3", (N_OUT, N_HID)), ("b3", (N_OUT,))):
        size = int(np.prod(shape))
        out[o:o + size] = np.asarray(g[name], np.float32).reshape(-1)
        o += size
    return out, loss


def dp_project(kappa, mu, p_thr, tan_phi, pmax, qmax, s0, s1, jp):
    """Wolper_Drucker_Prager (gpu_implementation5.cu:48-94) in principal
    space for one crushed particle: (changed, s0', s1', Jp_inv')."""
    je = s0 * s1
    p_tr = -(kappa / 2.0) * (je * je - 1.0)
    sq0, sq1 = s0 * s0, s1 * s1
    half = (sq0 + sq1) / 2
    f = mu / je
    sh0, sh1 = f * (sq0 - half), f * (sq1 - half)
    q_tr = SQRT2 * np.sqrt(sh0 * sh0 + sh1 * sh1)
    if p_tr < -p_thr or jp < 1:
        je_new = np.sqrt(2.0 * p_thr / kappa + 1.0)
        sn = np.sqrt(je_new)
        return True, sn, sn, jp * (je_new / je)
    q_n_1 = 0.0 if p_tr > pmax else min((p_tr + p_thr) * tan_phi, qmax)
    if q_tr >= q_n_1:
        z = sh0 * sh0 + sh1 * sh1
        n0, n1 = sh0, sh1
        if z > 0:
            nn = np.sqrt(z)
            n0, n1 = sh0 / nn, sh1 / nn
        ff = (q_n_1 / SQRT2) * (je / mu)
        mean = (sq0 + sq1) / 2.0
        return True, np.sqrt(ff * n0 + mean), np.sqrt(ff * n1 + mean), jp
    return False, s0, s1, jp


def features(kappa, tan_phi, qmax, s0, s1, jp):
    return np.array([1e3 * (s0 - 1.0), 1e3 * (s1 - 1.0), 1e2 * (jp - 1.0), kappa * 1e-9, tan_phi, qmax * 1e-7],
                    dtype=np.float32)


def targets(s0, s1, jp, s0n, s1n, jpn):
    return np.array([1e3 * (s0n - s0), 1e3 * (s1n - s1), 1e2 * (jpn - jp)], dtype=np.float32)


def material(p):
    """The constants the projection depends on, from a SimParams."""
    return dict(kappa=p.kappa, mu=p.mu, p_thr=p.DP_threshold_p, tan_phi=p.DP_tan_phi, pmax=p.IceCompressiveStrength,
                qmax=p.IceShearStrength)


def synthetic_pairs(p, n, seed=0):
    """Labelled pairs from trial states spread around the crushed states
    of an indentation: stretches within +-4e-3 of 1, Jp_inv within
    [0.995, 1.02]."""
    m = material(p)
    rng = np.random.default_rng(seed)
    x = np.zeros((n, N_IN), np.float32)
    y = np.zeros((n, N_OUT), np.float32)
    for i in range(n):
        a, b = 1.0 + rng.uniform(-4e-3, 4e-3, 2)
        s0, s1 = max(a, b), min(a, b)
        jp = rng.uniform(0.995, 1.02)
        _, s0n, s1n, jpn = dp_project(m["kappa"], m["mu"], m["p_thr"], m["tan_phi"], m["pmax"], m["qmax"], s0, s1, jp)
        x[i] = features(m["kappa"], m["tan_phi"], m["qmax"], s0, s1, jp)
        y[i] = targets(s0, s1, jp, s0n, s1n, jpn)
    return x, y


def loss(net, x, t, exact=False):
    p = unpack(net)
    tn = (np.asarray(t, np.float32) - p["y_mu"]) / p["y_sd"]
    d = forward(net, x, exact=exact).astype(np.float64) - tn
    return float(np.sum(d * d) / (3 * len(x)))
