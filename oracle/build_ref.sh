#!/bin/sh
# Builds oracle/_ref/libref_svd.so from the reference's own SVD headers
# (simulation/helper_math.cuh, simulation/givens.cuh) where they lie under
# the read-only reference checkout. Test infrastructure only. The rest of
# the reference (Eigen, HDF5, cxxopts, Qt/VTK, CMake) is not buildable here.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${ICEMPM_REFERENCE:-/root/reference}
if [ ! -f "$REF/simulation/helper_math.cuh" ]; then
    echo "reference sources not found at $REF; skipping oracle/_ref" >&2
    exit 0
fi
mkdir -p "$HERE/_ref"
g++ -O2 -std=c++17 -fPIC -shared -w \
    -I"$HERE/ref_stub" -I/usr/local/cuda/include -I"$REF/simulation" \
    "$HERE/ref_svd_harness.cpp" -o "$HERE/_ref/libref_svd.so"
echo "built $HERE/_ref/libref_svd.so"
