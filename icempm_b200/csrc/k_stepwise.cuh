// k_stepwise.cuh -- the three substep kernels on the reference's own data
// layout, one launch each, FP64 throughout.
//
// These back the member-function API of GPU_Implementation5 (cuda_p2g,
// cuda_update_nodes, cuda_g2p; gpu_implementation5.cu:568-593) so that a
// caller that drives the substep kernel by kernel sees the reference's
// buffers: particle SoA of 16 pitched double rows, grid of 3 pitched double
// rows (mass, momentum x|velocity x, momentum y|velocity y), 100 angular
// force bins. SimParams is passed by value (it sits in the kernel-parameter
// constant bank, which is what __constant__ gprms was for).
//
// Kernel correspondence:
//   k_p2g_ref64     v2_kernel_p2g           gpu_implementation5.cu:148-213
//   k_update_ref64  v2_kernel_update_nodes  gpu_implementation5.cu:215-290
//   k_g2p_ref64     v2_kernel_g2p           gpu_implementation5.cu:294-379
// Out-of-grid stencil nodes raise the error word and are skipped (the
// reference raises gpu_error_indicator but still adds at the bad index).
#pragma once
#include "mpm_math64.cuh"

namespace icm {

__device__ __forceinline__ double *pts_row(const icy_SimParams &P, int r) { return P.pts_array + (size_t)r * P.nPtsPitch; }

__global__ void k_p2g_ref64(const icy_SimParams P, int *err)
{
    int pt = blockIdx.x * blockDim.x + threadIdx.x;
    if (pt >= P.nPts) return;
    const double dt = P.InitialTimeStep, vol = P.ParticleVolume, h = P.cellsize;
    const double m = P.ParticleMass;
    const size_t gp = P.nGridPitch;
    double x = pts_row(P, ICM_IDX_POSX)[pt], y = pts_row(P, ICM_IDX_POSX + 1)[pt];
    double v0 = pts_row(P, ICM_IDX_VELX)[pt], v1 = pts_row(P, ICM_IDX_VELX + 1)[pt];
    M2d F = {pts_row(P, ICM_IDX_FE00)[pt], pts_row(P, ICM_IDX_FE00 + 1)[pt], pts_row(P, ICM_IDX_FE00 + 2)[pt],
             pts_row(P, ICM_IDX_FE00 + 3)[pt]};
    M2d B = {pts_row(P, ICM_IDX_BP00)[pt], pts_row(P, ICM_IDX_BP00 + 1)[pt], pts_row(P, ICM_IDX_BP00 + 2)[pt],
             pts_row(P, ICM_IDX_BP00 + 3)[pt]};
    M2d tau = kirchhoff64(F, P.mu, P.kappa);
    double c = (dt * vol) * P.Dp_inv;
    double s00 = m * B.a00 - c * tau.a00, s01 = m * B.a01 - c * tau.a01;
    double s10 = m * B.a10 - c * tau.a10, s11 = m * B.a11 - c * tau.a11;
    Stencil64 st = stencil64(x, y, P.cellsize_inv);
    bool bad = false;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            double W = st.wx[i] * st.wy[j];
            double d0 = (i - st.fx) * h, d1 = (j - st.fy) * h;
            double incV0 = W * (v0 * m + (s00 * d0 + s01 * d1));
            double incV1 = W * (v1 * m + (s10 * d0 + s11 * d1));
            double incM = W * m;
            int i2 = i + st.bx, j2 = j + st.by;
            if (i2 < 0 || j2 < 0 || i2 >= P.GridX || j2 >= P.GridY) {
                bad = true;
                continue;
            }
            size_t idx = (size_t)i2 + (size_t)j2 * P.GridX;
            atomicAdd(&P.grid_array[idx], incM);
            atomicAdd(&P.grid_array[gp + idx], incV0);
            atomicAdd(&P.grid_array[2 * gp + idx], incV1);
        }
    if (bad) *err = 1;
}

// force_total (may be null): 2 doubles receiving this launch's summed reaction.
__global__ void k_update_ref64(const icy_SimParams P, double ind_x, double ind_y, double *force_total)
{
    int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= P.GridTotal) return;
    double mass = P.grid_array[idx];
    if (mass == 0) return;
    const size_t gp = P.nGridPitch;
    int ix = idx % P.GridX, iy = idx / P.GridX;
    NodeOut o = update_node64(P, ix, iy, mass, P.grid_array[gp + idx], P.grid_array[2 * gp + idx], ind_x, ind_y);
    if (o.bin >= 0) {
        atomicAdd(&P.indenter_force_accumulator[2 * o.bin], o.f0);
        atomicAdd(&P.indenter_force_accumulator[2 * o.bin + 1], o.f1);
        if (force_total) {
            atomicAdd(&force_total[0], o.f0);
            atomicAdd(&force_total[1], o.f1);
        }
    }
    P.grid_array[gp + idx] = o.v0;
    P.grid_array[2 * gp + idx] = o.v1;
}

__global__ void k_g2p_ref64(const icy_SimParams P, int recordPQ)
{
    int pt = blockIdx.x * blockDim.x + threadIdx.x;
    if (pt >= P.nPts) return;
    const size_t gp = P.nGridPitch;
    const double h_inv = P.cellsize_inv, dt = P.InitialTimeStep;
    double x = pts_row(P, ICM_IDX_POSX)[pt], y = pts_row(P, ICM_IDX_POSX + 1)[pt];
    M2d F = {pts_row(P, ICM_IDX_FE00)[pt], pts_row(P, ICM_IDX_FE00 + 1)[pt], pts_row(P, ICM_IDX_FE00 + 2)[pt],
             pts_row(P, ICM_IDX_FE00 + 3)[pt]};
    uint8_t *crushed_row = (uint8_t *)P.pts_array;
    const short *grain_row = (const short *)((const char *)P.pts_array + P.nPtsPitch);
    uint8_t crushed = crushed_row[pt];
    int grain = grain_row[pt];
    double Jp = pts_row(P, ICM_IDX_JP_INV)[pt];

    Stencil64 st = stencil64(x, y, h_inv);
    double v0 = 0, v1 = 0, B00 = 0, B01 = 0, B10 = 0, B11 = 0;
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            double d0 = i - st.fx, d1 = j - st.fy;
            double W = st.wx[i] * st.wy[j];
            int i2 = i + st.bx, j2 = j + st.by;
            double n0 = 0, n1 = 0;
            if (i2 >= 0 && j2 >= 0 && i2 < P.GridX && j2 < P.GridY) {
                size_t idx = (size_t)i2 + (size_t)j2 * P.GridX;
                n0 = P.grid_array[gp + idx];
                n1 = P.grid_array[2 * gp + idx];
            }
            v0 += W * n0;
            v1 += W * n1;
            double c = (4. * h_inv) * W;
            B00 += c * (n0 * d0);
            B01 += c * (n0 * d1);
            B10 += c * (n1 * d0);
            B11 += c * (n1 * d1);
        }
    x += v0 * dt;
    y += v1 * dt;
    double M00 = 1 + dt * B00, M01 = dt * B01, M10 = dt * B10, M11 = 1 + dt * B11;
    M2d Fn = {M00 * F.a00 + M01 * F.a10, M00 * F.a01 + M01 * F.a11, M10 * F.a00 + M11 * F.a10,
              M10 * F.a01 + M11 * F.a11};
    double p_tr, q_tr;
    constitutive64(P, Fn, Jp, crushed, grain_res(grain), p_tr, q_tr);

    pts_row(P, ICM_IDX_JP_INV)[pt] = Jp;
    pts_row(P, ICM_IDX_POSX)[pt] = x;
    pts_row(P, ICM_IDX_POSX + 1)[pt] = y;
    pts_row(P, ICM_IDX_VELX)[pt] = v0;
    pts_row(P, ICM_IDX_VELX + 1)[pt] = v1;
    pts_row(P, ICM_IDX_FE00)[pt] = Fn.a00;
    pts_row(P, ICM_IDX_FE00 + 1)[pt] = Fn.a01;
    pts_row(P, ICM_IDX_FE00 + 2)[pt] = Fn.a10;
    pts_row(P, ICM_IDX_FE00 + 3)[pt] = Fn.a11;
    pts_row(P, ICM_IDX_BP00)[pt] = B00;
    pts_row(P, ICM_IDX_BP00 + 1)[pt] = B01;
    pts_row(P, ICM_IDX_BP00 + 2)[pt] = B10;
    pts_row(P, ICM_IDX_BP00 + 3)[pt] = B11;
    crushed_row[pt] = crushed;
    if (recordPQ) {
        pts_row(P, ICM_IDX_P)[pt] = p_tr;
        pts_row(P, ICM_IDX_Q)[pt] = q_tr;
    }
}

}  // namespace icm
