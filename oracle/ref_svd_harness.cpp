// ref_svd_harness.cpp -- compiles the reference's own 2x2 SVD
// (simulation/helper_math.cuh:81-140 with simulation/givens.cuh) for the host
// and exports it through C. TEST INFRASTRUCTURE: used only by tests/ to pin
// the oracle's SVD restatement. Built by oracle/build_ref.sh into
// oracle/_ref/; nothing of the reference is copied into this repository.
//
// helper_math.cuh pulls in parameters_sim.h and point.h (Eigen, rapidjson)
// but uses nothing from them: their include guards are pre-defined here and
// <Eigen/Core> resolves to an empty stub (oracle/ref_stub). Under g++ the
// __device__ qualifiers from cuda_runtime.h are inert, so the device
// functions compile as host functions.
#define P_SIM_H
#define PARTICLE_H
#include "helper_math.cuh"

// The glue of gpu_implementation5.cu:399-406 (svd): identity rotations in,
// singular_value_decomposition, then fill<2> of both rotations.
extern "C" void ref_svd(const double a[4], double u[4], double sigma[2], double v[4])
{
    GivensRotation<double> gv(0, 1);
    GivensRotation<double> gu(0, 1);
    singular_value_decomposition(a, gu, sigma, gv);
    gu.template fill<2, double>(u);
    gv.template fill<2, double>(v);
}
