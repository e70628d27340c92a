// ref_step_harness.cpp -- exports the reference's own substep code, compiled
// for the host, through C. TEST INFRASTRUCTURE: used only by tests/ to pin
// the oracle (oracle/mpm_oracle.c) to the reference, function by function
// and substep by substep.
//
// oracle/build_ref.sh compiles two translation units into
// oracle/_ref/libref_step.so: lines 1-416 of the reference's
// simulation/gpu_implementation5.cu (read from the reference checkout and
// piped to g++; nothing of it is copied into this repository) -- gprms,
// gpu_error_indicator, KirchhoffStress_Wolper, ComputePQ,
// Wolper_Drucker_Prager, GetParametersForGrain,
// CheckIfPointIsInsideFailureSurface, v2_kernel_p2g, v2_kernel_update_nodes,
// v2_kernel_g2p, dev_d, dev, svd, svd2x2_modified -- and this file. Both are
// prefixed with ref_step_pre.h (host stand-ins for the CUDA built-ins) and
// see the Eigen subset of oracle/ref_stub.
//
// Every entry point takes the run's parameter block in this project's
// icy_SimParams layout (include/icempm_params.h), which is byte for byte the
// reference's icy::SimParams (ref_params_size() lets a test check the size),
// and copies it into gprms first, as cuda_update_constants does
// (gpu_implementation5.cu:471-479).
#include <cstring>

#include "gpu_implementation5.h"

extern icy::SimParams gprms;
extern int gpu_error_indicator;

uint3 ref_thread_idx, ref_block_idx;
dim3 ref_block_dim;

double atomicAdd(double *address, double val)
{
    const double old = *address;
    *address = old + val;
    return old;
}

namespace {

void set_params(const void *p) { std::memcpy(&gprms, p, sizeof(gprms)); }

void set_index(int i)
{
    ref_block_dim.x = 1;
    ref_block_idx.x = 0;
    ref_thread_idx.x = (unsigned)i;
}

Eigen::Matrix2d mat(const double a[4])
{
    Eigen::Matrix2d m;
    m << a[0], a[1], a[2], a[3];
    return m;
}

void put(const Eigen::Matrix2d &m, double a[4])
{
    a[0] = m(0, 0);
    a[1] = m(0, 1);
    a[2] = m(1, 0);
    a[3] = m(1, 1);
}

}  // namespace

extern "C" int ref_params_size(void) { return (int)sizeof(icy::SimParams); }

// KirchhoffStress_Wolper (gpu_implementation5.cu:24-34); F, tau row-major.
extern "C" void ref_kirchhoff(const void *params, const double F[4], double tau[4])
{
    set_params(params);
    put(KirchhoffStress_Wolper(mat(F)), tau);
}

// ComputePQ (:36-44). out: U[4], sigma[2], V[4] (row-major, as
// svd2x2_modified fills them), Je_tr, p_tr, q_tr, vSigmaSquared[2],
// v_s_hat_tr[2] -- 17 doubles.
extern "C" void ref_compute_pq(const void *params, const double F[4], double out[17])
{
    set_params(params);
    icy::Point p;
    p.Fe = mat(F);
    ComputePQ(p, gprms.kappa, gprms.mu);
    put(p.U, out);
    out[4] = p.vSigma[0];
    out[5] = p.vSigma[1];
    put(p.V, out + 6);
    out[10] = p.Je_tr;
    out[11] = p.p_tr;
    out[12] = p.q_tr;
    out[13] = p.vSigmaSquared[0];
    out[14] = p.vSigmaSquared[1];
    out[15] = p.v_s_hat_tr[0];
    out[16] = p.v_s_hat_tr[1];
}

// GetParametersForGrain (:97-111). out: pmin, pmax, qmax, beta, mSq.
extern "C" void ref_grain_params(const void *params, short grain, double out[5])
{
    set_params(params);
    GetParametersForGrain(grain, out[0], out[1], out[2], out[3], out[4]);
}

// CheckIfPointIsInsideFailureSurface (:114-141) for an intact point with the
// given trial p, q; returns the new crushed flag.
extern "C" int ref_failure_check(const void *params, short grain, double p_tr, double q_tr)
{
    set_params(params);
    icy::Point p;
    p.grain = grain;
    p.crushed = 0;
    p.p_tr = p_tr;
    p.q_tr = q_tr;
    CheckIfPointIsInsideFailureSurface(p);
    return p.crushed;
}

// The constitutive part of v2_kernel_g2p (:353-356): ComputePQ, the failure
// check for an intact point, Wolper_Drucker_Prager (:48-94) for a crushed
// one. Fe (row-major), Jp_inv and crushed are updated in place.
extern "C" void ref_constitutive(const void *params, double Fe[4], double *Jp_inv, unsigned char *crushed, short grain,
                                 double *p_tr, double *q_tr)
{
    set_params(params);
    icy::Point p;
    p.Fe = mat(Fe);
    p.Jp_inv = *Jp_inv;
    p.crushed = *crushed;
    p.grain = grain;
    ComputePQ(p, gprms.kappa, gprms.mu);
    if (p.crushed == 0) CheckIfPointIsInsideFailureSurface(p);
    if (p.crushed == 1) Wolper_Drucker_Prager(p);
    put(p.Fe, Fe);
    *Jp_inv = p.Jp_inv;
    *crushed = p.crushed;
    *p_tr = p.p_tr;
    *q_tr = p.q_tr;
}

// n substeps of icy::Model::Step's loop (model.cpp:20-29) over the
// reference's three kernels, each kernel body called once per particle or
// node in index order: reset grid (cuda_reset_grid), v2_kernel_p2g,
// v2_kernel_update_nodes(indenter_x, indenter_y), v2_kernel_g2p(recordPQ).
// pts: the 16-row pitched SoA (nPtsPitch doubles per row); grid: 3 rows of
// nGridPitch doubles; bins: 2 * n_indenter_subdivisions doubles, accumulated
// (the caller resets them per frame). SimulationStep, SimulationTime and
// indenter_x of *params advance as Model::Step advances them. Returns
// gpu_error_indicator.
extern "C" int ref_run_substeps(void *params, double *pts, double *grid, double *bins, int n)
{
    icy::SimParams prms;
    std::memcpy(&prms, params, sizeof(prms));
    prms.pts_array = pts;
    prms.grid_array = grid;
    prms.indenter_force_accumulator = bins;
    set_params(&prms);
    gpu_error_indicator = 0;
    double simulation_time = prms.SimulationTime;
    for (int k = 1; k <= n; k++) {
        simulation_time += prms.InitialTimeStep;
        prms.indenter_x = prms.indenter_x_initial + simulation_time * prms.IndVelocity;
        std::memset(grid, 0, sizeof(double) * prms.nGridPitch * icy::SimParams::nGridArrays);
        for (int i = 0; i < prms.nPts; i++) {
            set_index(i);
            v2_kernel_p2g();
        }
        for (int i = 0; i < prms.GridTotal; i++) {
            set_index(i);
            v2_kernel_update_nodes(prms.indenter_x, prms.indenter_y);
        }
        const bool record = (prms.SimulationStep + k) % prms.UpdateEveryNthStep == 0;
        for (int i = 0; i < prms.nPts; i++) {
            set_index(i);
            v2_kernel_g2p(record);
        }
    }
    icy::SimParams *out = static_cast<icy::SimParams *>(params);
    out->SimulationStep = prms.SimulationStep + n;
    out->SimulationTime = simulation_time;
    out->indenter_x = prms.indenter_x;
    return gpu_error_indicator;
}
