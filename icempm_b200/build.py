"""Builds the in-tree native libraries.

* ``icempm_b200/libicempm.so`` -- the CUDA kernels (sm_100a) and the C ABI of
  ``include/icempm.h``, compiled with nvcc.
* ``icempm_b200/cm`` -- the C++ command-line driver (``cli/cm.cpp``), built on
  the C++ shim ``include/icempm.hpp``.

The checker libraries under ``oracle/`` are built by ``build_oracle`` (test
infrastructure; the package never loads them).

Run ``python -m icempm_b200.build`` or call :func:`build_all`.
"""
from __future__ import annotations

import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libicempm.so")
CLI = os.path.join(PKG, "cm")
ORACLE = os.path.join(ROOT, "oracle")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CU_SOURCES = ["device_layer.cu", "noalloc.cu", "mlp.cu"]
CPP_SOURCES = ["params.cpp", "scene.cpp", "errors.cpp", "snapshot.cpp", "hdf5_lite.cpp"]


def _deps():
    out = []
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".cu", ".cuh", ".cpp", ".h", ".hpp")):
                out.append(os.path.join(d, f))
    return out


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd, cwd=None):
    r = subprocess.run(cmd, cwd=cwd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("build failed: " + " ".join(cmd))
    return r


def build_lib(force: bool = False) -> str:
    """Compiles libicempm.so for sm_100a (nvcc cross-compiles without a GPU)."""
    srcs = [os.path.join(CSRC, s) for s in CU_SOURCES + CPP_SOURCES if os.path.exists(os.path.join(CSRC, s))]
    if not force and not _stale(LIB, _deps()):
        return LIB
    cmd = ["nvcc", *ARCH, "-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
           "-o", LIB + ".tmp", *srcs, "-lz"]
    _run(cmd)
    os.replace(LIB + ".tmp", LIB)
    return LIB


def build_cli(force: bool = False) -> str:
    """Builds the C++ driver against libicempm.so."""
    src = os.path.join(PKG, "cli", "cm.cpp")
    if not os.path.exists(src):
        return ""
    if not force and not _stale(CLI, _deps() + [src, LIB]):
        return CLI
    cmd = ["g++", "-O2", "-std=c++17", "-pthread", "-Wall", "-I", os.path.join(ROOT, "include"), src,
           "-L", PKG, "-licempm", "-Wl,-rpath,$ORIGIN", "-o", CLI]
    _run(cmd)
    return CLI


def build_oracle(force: bool = False) -> None:
    """Builds the CPU oracle and, when the reference checkout is present, the
    reference's own SVD and substep code for the host (oracle/_ref; test
    infrastructure)."""
    target = os.path.join(ORACLE, "libmpm_oracle.so")
    if force or _stale(target, [os.path.join(ORACLE, "mpm_oracle.c"), os.path.join(ORACLE, "scene_oracle.c"),
                                os.path.join(ROOT, "include", "icempm_params.h")]):
        _run(["make", "-C", ORACLE, "libmpm_oracle.so"] + (["-B"] if force else []))
    refs = [os.path.join(ORACLE, "_ref", f) for f in ("libref_svd.so", "libref_step.so")]
    srcs = [os.path.join(ORACLE, f) for f in ("build_ref.sh", "ref_svd_harness.cpp", "ref_step_harness.cpp",
                                               "ref_step_pre.h", os.path.join("ref_stub", "Eigen", "Core"))]
    if force or any(_stale(r, srcs) for r in refs):
        _run(["sh", os.path.join(ORACLE, "build_ref.sh")])


def build_all(force: bool = False) -> None:
    build_lib(force)
    build_cli(force)
    build_oracle(force)


if __name__ == "__main__":
    build_all(force="--force" in sys.argv)
    print("built", LIB)
