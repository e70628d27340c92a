// ref_step_pre.h -- force-included (g++ -include) ahead of the reference's
// simulation/gpu_implementation5.cu (its device part, lines 1-416) and of
// ref_step_harness.cpp when oracle/build_ref.sh builds oracle/_ref/
// libref_step.so. TEST INFRASTRUCTURE: host stand-ins for what the device
// code takes from the CUDA compiler.
//
// * __device__, __global__ and __constant__ come from cuda_runtime.h, where
//   they are inert under g++: the kernels become host functions and gprms a
//   host global.
// * threadIdx / blockIdx / blockDim name host variables that the harness
//   sets before each call of a kernel body (one "thread" per call).
// * atomicAdd(double *, double) is a plain addition: the harness calls the
//   kernel bodies one after another, in index order.
// * min / max are the std ones (the device code calls them on int and
//   double).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>

using std::max;
using std::min;

extern uint3 ref_thread_idx, ref_block_idx;
extern dim3 ref_block_dim;
#define threadIdx ref_thread_idx
#define blockIdx ref_block_idx
#define blockDim ref_block_dim

double atomicAdd(double *address, double val);
