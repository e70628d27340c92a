"""Generates the committed golden fixtures of tests/golden/.

* svd_ref.npz -- inputs and outputs of the reference's OWN 2x2 SVD
  (simulation/helper_math.cuh + givens.cuh compiled for the host by
  oracle/build_ref.sh into oracle/_ref/libref_svd.so). Pins the oracle's SVD
  restatement on machines without the reference checkout.
* oracle_small.npz -- a small perturbed block scene and its state after
  8 substeps of the oracle (1 thread): a regression pin of the oracle.

Run from the repository root: python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import oracle as orc  # noqa: E402
from tests.mpm_cases import params, scene, oracle_run  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))


def svd_inputs(rng):
    mats = []
    for _ in range(192):
        mats.append(rng.standard_normal(4))
    for _ in range(128):
        mats.append(np.array([1.0, 0.0, 0.0, 1.0]) + 1e-3 * rng.standard_normal(4))
    for _ in range(64):
        a = rng.standard_normal(4)
        a[2] = a[1]
        mats.append(a)
    for _ in range(32):
        d = rng.standard_normal(2)
        mats.append(np.array([d[0], 0.0, 0.0, d[1]]))  # y2 == 0 path
    for _ in range(32):
        a = rng.standard_normal(4)
        a[0], a[1] = -a[0], -a[1]  # negative determinants
        mats.append(a)
    for _ in range(32):
        th = rng.uniform(-np.pi, np.pi)
        s = rng.uniform(0.5, 2)
        mats.append(s * np.array([np.cos(th), -np.sin(th), np.sin(th), np.cos(th)]))  # repeated sigma
    mats.append(np.zeros(4))
    mats.append(np.array([1.0, 0.0, 0.0, 1.0]))
    mats.append(np.array([0.0, 1.0, -1.0, 0.0]))
    mats.append(np.array([2.0, 0.0, 0.0, -3.0]))
    return np.array(mats)


def main():
    rng = np.random.default_rng(20241203)
    ref = orc.ref_svd_lib()
    if ref is None:
        raise SystemExit("oracle/_ref/libref_svd.so not built (run oracle/build_ref.sh)")
    A = svd_inputs(rng)
    U = np.zeros_like(A)
    S = np.zeros((len(A), 2))
    V = np.zeros_like(A)
    for k, a in enumerate(A):
        a = np.ascontiguousarray(a)
        u, s, v = np.zeros(4), np.zeros(2), np.zeros(4)
        ref.ref_svd(a.ctypes.data, u.ctypes.data, s.ctypes.data, v.ctypes.data)
        U[k], S[k], V[k] = u, s, v
    np.savez_compressed(os.path.join(HERE, "svd_ref.npz"), A=A, U=U, S=S, V=V)

    p = params(64, 32, 0.5, 2e-6)
    soa = scene(p, cells=(24, 8), seed=11, ind_y=0.03, perturb=2e-3, vel=0.05, crushed_frac=0.3, jp_spread=0.01)
    q, out, bins, err, hist = oracle_run(p, soa, 8, threads=1)
    np.savez_compressed(os.path.join(HERE, "oracle_small.npz"), params=np.frombuffer(p.to_bytes(), np.uint8),
                        soa_in=soa, soa_out=out, bins=bins, hist=hist, err=err,
                        params_out=np.frombuffer(q.to_bytes(), np.uint8))
    print("wrote", len(A), "SVD cases and an 8-substep oracle run of", p.nPts, "particles")


if __name__ == "__main__":
    main()
