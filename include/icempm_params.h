/*
 * icempm_params.h -- the simulation parameter block shared by the host, the
 * CUDA kernels and the snapshot format.
 *
 * Byte-for-byte the layout of icy::SimParams (simulation/parameters_sim.h:19-90
 * in iceMPM). The reference copies the struct raw into __constant__ memory
 * (gpu_implementation5.cu:476) and into the `Params` dataset of every snapshot
 * (snapshotmanager.cpp:80-83), so the field order, the types and the padding
 * are part of the file format and are kept exactly. The offsets are checked
 * with static asserts below (x86-64 / LP64, the only ABI both sides run on).
 *
 * Device pointers (grid_array, indenter_force_accumulator, pts_array) live
 * inside the struct as in the reference; pitches are counted in doubles.
 */
#ifndef ICEMPM_PARAMS_H
#define ICEMPM_PARAMS_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Row indices of the particle structure-of-arrays (parameters_sim.h:27-35).
 * Row 0 holds bytes: crushed flag (u8) at byte i, grain id (i16) at byte
 * offset pitch*1 + 2*i of the row block (point.cpp:19-23). */
enum {
    ICM_IDX_UTILITY = 0,
    ICM_IDX_P = 1,
    ICM_IDX_Q = 2,
    ICM_IDX_JP_INV = 3,
    ICM_IDX_POSX = 4,
    ICM_IDX_VELX = 6,
    ICM_IDX_FE00 = 8,
    ICM_IDX_BP00 = 12,
    ICM_N_PTS_ARRAYS = 16,
    ICM_N_GRID_ARRAYS = 3,
    ICM_DIM = 2
};

#define ICM_PI 3.14159265358979323846

typedef struct icy_SimParams {
    double *grid_array;                 /* device grid, 3 pitched rows: m, px|vx, py|vy */
    double *indenter_force_accumulator; /* device, 2*n_indenter_subdivisions doubles */
    double *pts_array;                  /* device particle SoA, 16 pitched rows */

    size_t nPtsPitch, nGridPitch;       /* in elements (doubles) */
    int n_indenter_subdivisions;
    int tpb_P2G, tpb_Upd, tpb_G2P;

    int nPts;
    int GridX, GridY, GridTotal;
    double GridXDimension;

    double InitialTimeStep, SimulationEndTime;
    double Gravity, Density, PoissonsRatio, YoungsModulus;
    double lambda, mu, kappa;

    double IceCompressiveStrength, IceTensileStrength, IceShearStrength;
    double NACC_beta, NACC_M, NACC_Msq;

    double DP_tan_phi, DP_threshold_p;

    double cellsize, cellsize_inv, Dp_inv;

    int UpdateEveryNthStep;

    double IndDiameter, IndRSq, IndVelocity, IndDepth;
    double xmin, xmax, ymin, ymax;
    int nxmin, nxmax, nymin, nymax;

    double ParticleVolume, ParticleMass, ParticleViewSize;

    int SimulationStep;
    double SimulationTime;

    double indenter_x, indenter_x_initial, indenter_y, indenter_y_initial;
    double Volume;
    int SetupType;
    double GrainVariability;

    int UseWarpLevelReduction;
    int SortPointsByGridCell;
} icy_SimParams;

#ifdef __cplusplus
} /* extern "C" */

#define ICM_CHECK_OFFSET(field, off) \
    static_assert(offsetof(icy_SimParams, field) == (off), "SimParams layout: " #field)
ICM_CHECK_OFFSET(grid_array, 0);
ICM_CHECK_OFFSET(indenter_force_accumulator, 8);
ICM_CHECK_OFFSET(pts_array, 16);
ICM_CHECK_OFFSET(nPtsPitch, 24);
ICM_CHECK_OFFSET(nGridPitch, 32);
ICM_CHECK_OFFSET(n_indenter_subdivisions, 40);
ICM_CHECK_OFFSET(tpb_P2G, 44);
ICM_CHECK_OFFSET(nPts, 56);
ICM_CHECK_OFFSET(GridX, 60);
ICM_CHECK_OFFSET(GridTotal, 68);
ICM_CHECK_OFFSET(GridXDimension, 72);
ICM_CHECK_OFFSET(InitialTimeStep, 80);
ICM_CHECK_OFFSET(Gravity, 96);
ICM_CHECK_OFFSET(lambda, 128);
ICM_CHECK_OFFSET(kappa, 144);
ICM_CHECK_OFFSET(IceCompressiveStrength, 152);
ICM_CHECK_OFFSET(NACC_beta, 176);
ICM_CHECK_OFFSET(DP_tan_phi, 200);
ICM_CHECK_OFFSET(DP_threshold_p, 208);
ICM_CHECK_OFFSET(cellsize, 216);
ICM_CHECK_OFFSET(Dp_inv, 232);
ICM_CHECK_OFFSET(UpdateEveryNthStep, 240);
ICM_CHECK_OFFSET(IndDiameter, 248);
ICM_CHECK_OFFSET(IndVelocity, 264);
ICM_CHECK_OFFSET(xmin, 280);
ICM_CHECK_OFFSET(nxmin, 312);
ICM_CHECK_OFFSET(ParticleVolume, 328);
ICM_CHECK_OFFSET(ParticleMass, 336);
ICM_CHECK_OFFSET(SimulationStep, 352);
ICM_CHECK_OFFSET(SimulationTime, 360);
ICM_CHECK_OFFSET(indenter_x, 368);
ICM_CHECK_OFFSET(indenter_y, 384);
ICM_CHECK_OFFSET(Volume, 400);
ICM_CHECK_OFFSET(SetupType, 408);
ICM_CHECK_OFFSET(GrainVariability, 416);
ICM_CHECK_OFFSET(UseWarpLevelReduction, 424);
ICM_CHECK_OFFSET(SortPointsByGridCell, 428);
static_assert(sizeof(icy_SimParams) == 432, "SimParams must be 432 bytes");
#undef ICM_CHECK_OFFSET
#endif

#endif /* ICEMPM_PARAMS_H */
