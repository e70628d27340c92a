#!/bin/sh
# Builds the checker libraries of oracle/_ref/ from the reference's own
# sources, where they lie in the read-only reference checkout (location:
# $ICEMPM_REFERENCE, else the default below). TEST INFRASTRUCTURE only.
#
#   libref_svd.so   simulation/helper_math.cuh + givens.cuh (the 2x2 SVD)
#   libref_step.so  simulation/gpu_implementation5.cu lines 1-416: the device
#                   functions and the three kernel bodies, compiled for the
#                   host against the Eigen subset in ref_stub/ and the CUDA
#                   stand-ins of ref_step_pre.h (ref_step_harness.cpp)
#
# The source lines are piped to g++; nothing of the reference is written
# into this repository. The rest of the reference (HDF5, cxxopts, Qt/VTK,
# the CMake build, the host half of gpu_implementation5.cu with its kernel
# launches) is not built.
set -e
HERE=$(cd "$(dirname "$0")" && pwd)
REF=${ICEMPM_REFERENCE:-/root/reference}
SIM="$REF/simulation"
if [ ! -f "$SIM/helper_math.cuh" ] || [ ! -f "$SIM/gpu_implementation5.cu" ]; then
    echo "reference sources not found at $REF; skipping oracle/_ref" >&2
    exit 0
fi
mkdir -p "$HERE/_ref"
# where the sources were found, for tests that read the reference's data
# files (tests/conftest.py: reference_root)
printf '%s\n' "$REF" > "$HERE/_ref/reference_root"
g++ -O2 -std=c++17 -fPIC -shared -w \
    -I"$HERE/ref_stub" -I/usr/local/cuda/include -I"$SIM" \
    "$HERE/ref_svd_harness.cpp" -o "$HERE/_ref/libref_svd.so"
echo "built $HERE/_ref/libref_svd.so"

# the cut must end with svd2x2_modified (gpu_implementation5.cu:408-416);
# anything else means the reference changed and the line range is stale
if ! sed -n '408p' "$SIM/gpu_implementation5.cu" | grep -q 'svd2x2_modified' ||
   ! sed -n '416p' "$SIM/gpu_implementation5.cu" | grep -q '^}'; then
    echo "gpu_implementation5.cu:408-416 is not svd2x2_modified; libref_step.so not built" >&2
    exit 1
fi
sed -n '1,416p' "$SIM/gpu_implementation5.cu" |
    g++ -O2 -std=c++17 -fPIC -shared -w \
        -include "$HERE/ref_step_pre.h" -I"$HERE/ref_stub" -I/usr/local/cuda/include -I"$SIM" \
        -x c++ - -x c++ "$HERE/ref_step_harness.cpp" -o "$HERE/_ref/libref_step.so"
echo "built $HERE/_ref/libref_step.so"
