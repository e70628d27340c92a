/*
 * icempm.h -- C ABI of the B200 MLS-MPM substep library (libicempm.so).
 *
 * This is the drop-in boundary for iceMPM's device layer, the C++ class
 * GPU_Implementation5 (simulation/gpu_implementation5.h:40-72) and the step
 * loop that drives it (icy::Model::Step, simulation/model.cpp:11-47). Every
 * entry point takes plain pointers and sizes, returns ICM_OK (0) or an
 * ICM_ERR_* code and never throws; icm_last_error() gives the message of the
 * calling thread's last failure. The C++ shim in include/icempm.hpp turns a
 * non-zero status back into std::runtime_error, which is what the reference
 * members do (gpu_implementation5.cu:458-592).
 *
 * Buffers follow the reference:
 *   particles  16 rows x nPtsPitch doubles (parameters_sim.h:27-35), row 0
 *              holding the crushed byte at byte i and the grain id (int16)
 *              at byte offset nPtsPitch + 2*i (point.cpp:19-23);
 *   grid       3 rows x nGridPitch doubles: mass, momentum|velocity x, y;
 *   force bins 2*n_indenter_subdivisions doubles, accumulated over a frame.
 * Pitches are in elements and are written into SimParams by
 * icm_allocate_arrays, as cudaMallocPitch results are in the reference.
 */
#ifndef ICEMPM_H
#define ICEMPM_H

#include <stddef.h>
#include <stdint.h>
#include "icempm_params.h"

#ifdef __cplusplus
extern "C" {
#endif

enum {
    ICM_OK = 0,
    ICM_ERR_CUDA = 1,      /* a CUDA runtime call failed */
    ICM_ERR_ARG = 2,       /* bad argument (null pointer, size out of range) */
    ICM_ERR_STATE = 3,     /* call out of order (e.g. no arrays allocated) */
    ICM_ERR_NOMEM = 4,     /* device or host allocation failed */
    ICM_ERR_IO = 5,        /* file missing or unreadable */
    ICM_ERR_PARSE = 6,     /* configuration not valid JSON / missing key */
    ICM_ERR_NODEVICE = 7   /* no CUDA device */
};

/* Precision / execution forms of icm_run_substeps. */
enum {
    ICM_FORM_FP64_STEPWISE = 0, /* reference structure: reset, P2G, update, G2P launches per substep, FP64 */
    ICM_FORM_FP64 = 1,          /* fused tile substep, FP64 reference form */
    ICM_FORM_FP32 = 2,          /* fused tile substep, FP32 strain form */
    ICM_FORM_FP32_SURROGATE = 3, /* FP32 form with the learned Drucker-Prager projection (icm_set_surrogate) */
    ICM_FORM_FP32_COMPENSATED = 4 /* FP32 form with compensated (Kahan) per-cell momentum sums; single runs */
};

typedef struct icm_ctx icm_ctx;
typedef void (*icm_host_fn)(void *user);

const char *icm_last_error(void);
const char *icm_version(void);

/* ---------------------------------------------------------- SimParams
 * parameters_sim.cpp: Reset :5-56, ParseFile :59-119, ComputeLame :121-126,
 * ComputeHelperVariables :128-136, ComputeCamClayParams2 :138-147,
 * ComputeIntegerBlockCoords :149-155. */
void icm_params_reset(icy_SimParams *p);
/* Parses a flat JSON object (the keys of parameters_sim.cpp:73-99) and
 * recomputes the derived values. Copies "InputRawPoints" into raw_points
 * (may be NULL); returns ICM_ERR_PARSE if that key is missing, as ParseFile
 * throws "config parameter missing" (parameters_sim.cpp:110-114). */
int icm_params_parse_file(icy_SimParams *p, const char *path, char *raw_points, size_t cap);
int icm_params_parse_string(icy_SimParams *p, const char *json, char *raw_points, size_t cap);
void icm_params_compute_lame(icy_SimParams *p);
void icm_params_compute_camclay(icy_SimParams *p);
void icm_params_compute_helpers(icy_SimParams *p);
void icm_params_compute_block_coords(icy_SimParams *p);
/* Pitch (elements) used for an array of n doubles: n rounded up to 64. */
size_t icm_pitch_elems(size_t n);

/* ------------------------------------------------ synthetic ice block
 * Stands in for SnapshotManager::LoadRawPoints (snapshotmanager.cpp:186-286)
 * when no HDF5 point cloud is given: a block of cells_x x cells_y cells at
 * 2x2 jittered sites per cell (jitter +-0.25 sub-cell), seeded Voronoi grains
 * (about one per grain_size metres), sorted by grid cell as SortPoints does
 * (snapshotmanager.cpp:288-304). Sets nPts, Volume, bounding box,
 * ParticleVolume, ParticleMass and the indenter start: x = block_left - r,
 * y = block_bottom + ind_y_above_floor. Fills host_soa (16 x pitch doubles,
 * pitch = icm_pitch_elems(n)) when it is not NULL; returns the particle
 * count through n_out. */
typedef struct icm_block_desc {
    int cells_x, cells_y;       /* block size in grid cells */
    double ind_y_above_floor;   /* indenter centre above the block bottom, metres */
    double grain_size;          /* metres per Voronoi grain */
    uint64_t seed;
} icm_block_desc;
int icm_scene_block(icy_SimParams *p, const icm_block_desc *d, double *host_soa, int *n_out);

/* -------------------------------------------------------- device layer */

/* GPU_Implementation5::initialize (gpu_implementation5.cu:452-469). */
int icm_create(icm_ctx **out, int device);
/* Frees device and host buffers the context owns (the reference has no
 * destructor). */
int icm_destroy(icm_ctx *ctx);
/* Selects the form used by icm_run_substeps (an extension of SimParams'
 * role; the reference has only the FP64 stepwise form). */
int icm_set_form(icm_ctx *ctx, int form);
int icm_get_form(icm_ctx *ctx);
/* Tile shape of the fused forms: index into the built variants
 * (0: 16x8, 1: 16x16, 2: 32x8, 3: 32x16 nodes) and block size (default
 * 16x16 nodes, 128 threads). */
int icm_set_tile(icm_ctx *ctx, int tile_variant, int threads);
int icm_get_tile(icm_ctx *ctx, int *tile_variant, int *threads);
/* Fused forms: re-bin the particles by their current grid cell every
 * `substeps` substeps of a run of icm_run_substeps, counted from the run's
 * start and never after its last substep (default 100). 0: only when the
 * particles are packed (the first run after an upload or a change of form
 * or tile). Particles that left their binned cell take a slower scatter
 * path until then. */
int icm_set_rebin_interval(icm_ctx *ctx, int substeps);
/* Fused forms: a tile whose last measured cost exceeds `ratio` times the
 * mean over tiles holding particles runs as two CTAs (each half of its cell
 * groups), at most `max_tiles` tiles per launch; the heaviest tiles -- the
 * crushed zone at the indenter -- otherwise set the length of a launch late
 * in a frame. Default 128 tiles, ratio 1.3; max_tiles 0 turns it off. No
 * counterpart in the reference. */
int icm_set_tile_split(icm_ctx *ctx, int max_tiles, double ratio);
/* GPU_Implementation5::cuda_allocate_arrays (gpu_implementation5.cu:481-513):
 * device particle SoA, grid and force bins. Writes the device pointers and
 * pitches into *p and resets the error code. */
int icm_allocate_arrays(icm_ctx *ctx, icy_SimParams *p, size_t n_grid_nodes, size_t n_points);
/* GPU_Implementation5::cuda_update_constants (gpu_implementation5.cu:471-479):
 * takes a copy of *p for the kernels and writes error_code to the device
 * error word. */
int icm_update_constants(icm_ctx *ctx, const icy_SimParams *p, int error_code);
/* GPU_Implementation5::transfer_ponts_to_device (gpu_implementation5.cu:515-526). */
int icm_transfer_points_to_device(icm_ctx *ctx, const double *host_soa);
/* GPU_Implementation5::cuda_reset_grid (gpu_implementation5.cu:554-559). */
int icm_reset_grid(icm_ctx *ctx);
/* GPU_Implementation5::cuda_reset_indenter_force_accumulator (:561-565). */
int icm_reset_indenter_force_accumulator(icm_ctx *ctx);
/* GPU_Implementation5::cuda_p2g (gpu_implementation5.cu:568-575). */
int icm_p2g(icm_ctx *ctx);
/* GPU_Implementation5::cuda_update_nodes (gpu_implementation5.cu:577-584). */
int icm_update_nodes(icm_ctx *ctx, double indenter_x, double indenter_y);
/* GPU_Implementation5::cuda_g2p (gpu_implementation5.cu:586-593). */
int icm_g2p(icm_ctx *ctx, int record_pq);
/* GPU_Implementation5::cuda_transfer_from_device (gpu_implementation5.cu:528-544):
 * enqueues the copies of the particle SoA (host_soa may be NULL), the force
 * bins (host_bins may be NULL) and the error word, then the host function
 * cb(user) (the stream callback of :542-552; it must not call CUDA). The
 * copies complete asynchronously: call icm_synchronize or wait for cb. */
int icm_transfer_from_device(icm_ctx *ctx, double *host_soa, double *host_bins, int *error_code,
                             icm_host_fn cb, void *user);
/* Copies of the reference-layout grid (3 rows x nGridPitch doubles). The
 * reference keeps the grid private to its kernels; these serve callers and
 * tests that drive the member-style kernels one by one. Synchronous. */
int icm_transfer_grid_to_device(icm_ctx *ctx, const double *host_grid);
int icm_transfer_grid_from_device(icm_ctx *ctx, double *host_grid);
/* GPU_Implementation5::synchronize (gpu_implementation5.cu:442-446). */
int icm_synchronize(icm_ctx *ctx);
/* The substep loop of icy::Model::Step (model.cpp:20-29): n substeps of
 * t += dt; indenter_x = indenter_x_initial + t*IndVelocity; reset; P2G;
 * update; G2P, with P and Q recorded on every substep that ends a frame
 * ((SimulationStep + k) % UpdateEveryNthStep == 0). Runs in the form set by
 * icm_set_form, advances p->SimulationStep, SimulationTime and indenter_x,
 * and keeps each substep's summed indenter reaction (see
 * icm_force_history). Asynchronous on the context's stream. */
int icm_run_substeps(icm_ctx *ctx, icy_SimParams *p, int n);
/* Copies the per-substep reaction totals (2 doubles each) of the last
 * icm_run_substeps into host_out (synchronous). */
int icm_force_history(icm_ctx *ctx, double *host_out, int n);
/* Number of particles the FP32 form handed to the FP64 fallback since the
 * context was created (synchronous). */
int icm_fp64_redo_count(icm_ctx *ctx, unsigned long long *out);
/* Particle-substeps of the fused forms in which a particle's base node was
 * no longer the grid cell it was binned to (it then scatters through the
 * slower per-particle path); cumulative since the context was created
 * (synchronous). */
int icm_stray_count(icm_ctx *ctx, unsigned long long *out);
/* CUDA events around work on the context's stream (eventCycleStart/Stop of
 * gpu_implementation5.h:61). */
int icm_record_start(icm_ctx *ctx);
int icm_record_stop(icm_ctx *ctx);
int icm_elapsed_ms(icm_ctx *ctx, float *ms);
/* The two events above as cudaEvent_t handles, for callers that record
 * them themselves as model.cpp:19,30 does. */
int icm_cycle_events(icm_ctx *ctx, void **start, void **stop);
/* Per-launch timing of the fused substep kernel: when enabled, every
 * steady-state launch of icm_run_substeps is bracketed by a CUDA event pair
 * on the context's stream; icm_kernel_time returns the summed durations and
 * the launch count since enabling (synchronises). */
int icm_kernel_timing(icm_ctx *ctx, int enable);
int icm_kernel_time(icm_ctx *ctx, double *total_ms, long long *launches);
/* The context's CUDA stream (cudaStream_t) for callers that interleave
 * their own work. */
void *icm_stream(icm_ctx *ctx);
/* No counterpart in the reference. For callers that cannot allocate device
 * memory while they run -- an allocation can block or synchronise the whole
 * device, a host framework may own all GPU memory through its own pool, or
 * the caller works to a fixed memory budget -- this runs n substeps of the
 * FP64 step-wise form (the arithmetic of icm_run_substeps with
 * ICM_FORM_FP64_STEPWISE) on caller-owned device buffers and allocates
 * nothing: pts is the particle SoA (16 rows x p->nPtsPitch doubles, updated
 * in place), bins the 2*n_indenter_subdivisions force bins (accumulated),
 * err the error word (set to 1 when a stencil leaves the grid), stream a
 * cudaStream_t (NULL: the default stream). p is advanced as by
 * icm_run_substeps. The grid scratch is a fixed array inside the library:
 * GridX*GridY may be at most 262,144 nodes (6 MiB, held by every GPU that
 * loads the library until exit); larger grids are rejected with
 * ICM_ERR_ARG. All calls share that scratch, so calls that overlap on the
 * GPU race and must not be issued concurrently. Each call made outside
 * stream capture looks up the scratch's device address in the current
 * context (so a context re-created after cudaDeviceReset gets its own); a
 * call on a stream under capture reuses the address of the device's last
 * call, so make the first call on a device before any stream capture. */
int icm_run_substeps_noalloc(icy_SimParams *p, double *pts, double *bins, int *err, int n, void *stream);
/* ------------------------------------------------ learned projection
 * No counterpart in the reference. A 6 -> 64 -> 64 -> 3 GELU network
 * (BF16 weights, FP32 accumulation) predicts the Drucker-Prager projection
 * of a crushed particle (Wolper_Drucker_Prager, gpu_implementation5.cu:
 * 48-94) in principal space from its trial singular values and Jp_inv.
 * Parameters are icm_mlp_floats() floats: W1[64][6], b1[64], W2[64][64],
 * b2[64], W3[3][64], b3[3], then the input/output normalisation x_mu[6],
 * x_sd[6], y_mu[3], y_sd[3]. */
int icm_mlp_floats(void);
/* Sets the normalisation part of net from n samples (x: n x 6, y: n x 3). */
int icm_mlp_normalise(float *net, const float *x, const float *y, int n);
typedef struct icm_mlp_train_cfg {
    int steps;        /* Adam steps */
    int batch_tiles;  /* batch = 128 * batch_tiles samples, drawn at random each step */
    float lr;         /* peak learning rate (cosine decay to lr/20) */
    uint32_t seed;
} icm_mlp_train_cfg;
/* Trains net (in place; start from caller-initialised weights) on the
 * tensor cores of `device`; loss_hist (may be NULL) receives the mean
 * squared error of each step on normalised targets. */
int icm_mlp_train(int device, const float *x, const float *y, int n, const icm_mlp_train_cfg *cfg, float *net,
                  float *loss_hist);
/* Gradient of the mean squared error over the n samples (one forward and
 * backward pass of the training kernel) in the parameter layout, and the
 * loss. */
int icm_mlp_gradient(int device, const float *net, const float *x, const float *y, int n, float *grad, float *loss);
/* Network outputs (denormalised, n x 3) for n inputs: the tensor-core
 * batch form (warp_form = 0) or the warp form the substep uses (1). */
int icm_mlp_infer(int device, const float *net, const float *x, int n, float *y, int warp_form);
/* The surrogate form's network (NULL: none) and acceptance tolerance tau:
 * the network's projection of a crushed particle is used when it meets the
 * yield condition to within tau * IceShearStrength in q and tau * 1e-3 in
 * the stretches (the sum of squared stretches, i.e. the pressure, kept);
 * otherwise the exact projection runs. Resets the counters. */
int icm_set_surrogate(icm_ctx *ctx, const float *net, float tolerance);
/* Crushed-particle updates of the surrogate form since the network was
 * set: network projections accepted, and exact projections (rejected
 * predictions plus the hydrostatic branch, a closed form). */
int icm_surrogate_counts(icm_ctx *ctx, unsigned long long *accepted, unsigned long long *exact);
/* Training data: the fused FP32 forms record the trial state of every
 * crushed particle on substeps with (SimulationStep % every == 0), up to
 * capacity states (capacity or every 0: off). */
int icm_set_harvest(icm_ctx *ctx, int capacity, int every);
/* Labels the recorded states with the exact projection on the GPU and
 * returns up to cap pairs (features n x 6, targets n x 3); clears the
 * record. */
int icm_harvest_pairs(icm_ctx *ctx, const icy_SimParams *p, float *x, float *y, int cap, int *n_out);

/* ------------------------------------------------------------ ensembles
 * No counterpart in the reference. Many indentation cases -- each an
 * icm_ctx with its own block, material, indenter, grid and particle
 * arrays, set up as for icm_run_substeps -- advance together: every
 * substep is one launch over the active tiles of all cases (tiles holding
 * particles and their neighbours), the launches between re-binnings
 * replayed from a captured CUDA graph. Results per case are those of
 * icm_run_substeps on that case alone (same form and tile), up to the
 * order of float atomics: icm_force_history, icm_transfer_from_device etc.
 * read them from the case's context. */
typedef struct icm_ensemble icm_ensemble;
/* form: ICM_FORM_FP32, ICM_FORM_FP64 or ICM_FORM_FP32_SURROGATE (each case
 * with its own network from icm_set_surrogate; at most 128 threads);
 * tile_variant and threads as in icm_set_tile. */
int icm_ensemble_create(icm_ensemble **out, int device, int form, int tile_variant, int threads);
int icm_ensemble_destroy(icm_ensemble *e);
/* Adds a case (arrays allocated, points uploaded); sets its form and tile
 * to the ensemble's. The context stays the caller's. */
int icm_ensemble_add(icm_ensemble *e, icm_ctx *ctx);
int icm_ensemble_size(icm_ensemble *e);
/* Re-binning interval in substeps (default 200; 0: only when a run
 * starts) and whether segments are replayed from a CUDA graph (default 1). */
int icm_ensemble_set(icm_ensemble *e, int rebin_interval, int use_graphs);
/* n substeps of every case; p[i] is case i's SimParams, advanced as by
 * icm_run_substeps. Asynchronous: the cases' streams wait for it. A case
 * whose particles scattered into a tile outside its active set between two
 * re-binnings (mass that no launch consumed; a shorter re-binning interval
 * avoids it) gets bit 2 set in its error word (icm_transfer_from_device). */
int icm_ensemble_run(icm_ensemble *e, icy_SimParams *const *p, int n);
/* Heavy tiles of the launch list run as two CTAs, as icm_set_tile_split
 * (ratio to the mean over tiles with particles, across all cases). Default
 * off (max_tiles 0): a list of many cases has work enough that no single
 * tile sets the length of a launch. */
int icm_ensemble_set_split(icm_ensemble *e, int max_tiles, double ratio);
/* The ensemble's CUDA stream (cudaStream_t). */
void *icm_ensemble_stream(icm_ensemble *e);

/* ------------------------------------------------------------ snapshots
 * SnapshotManager (simulation/snapshotmanager.cpp) on the library's own
 * HDF5 reader and writer (no libhdf5); host-side, no device calls. Files
 * are numbered by the frame SimulationStep / UpdateEveryNthStep
 * (parameters_sim.h:88); path_out (may be NULL) receives the file written. */
/* SaveSnapshot (:60-104): <dir>/snapshots/d%05d.h5 with Indenter_2D
 * (f64[2*n_indenter_subdivisions]), Params (bitfield bytes[432], the
 * SimParams bytes, with the 14 attributes of SaveParametersAsAttributes
 * :106-142) and Points (f64[16*nPtsPitch], the particle SoA). */
int icm_save_snapshot(const icy_SimParams *p, const double *host_soa, const double *host_bins, const char *dir,
                      char *path_out, size_t cap);
/* Reading a snapshot back to resume a run (the reference's ReadSnapshot,
 * :145-184, is commented out): the stored SimParams (its device pointers
 * are the writer's and must be replaced), then the particle SoA (soa_elems
 * = 16*nPtsPitch) and force bins (host_bins may be NULL). */
int icm_read_snapshot_params(const char *path, icy_SimParams *out);
int icm_read_snapshot(const char *path, double *host_soa, size_t soa_elems, double *host_bins, size_t bins_elems);
/* SavePQ (:14-56): <dir>/pq/pq%05d.h5 with PQ_intact and PQ_crushed
 * (f64[n,2] of the P and Q rows, split by the crushed byte); PQ_intact
 * carries the parameter attributes. */
int icm_save_pq(const icy_SimParams *p, const double *host_soa, const char *dir, char *path_out, size_t cap);
/* LoadRawPoints (:186-286) + SortPoints (:288-304): reads Points_Raw_2D
 * (float[N,2]), GrainIDs (int16[N]) and its attribute volume (float), sorts
 * by grid cell when SortPointsByGridCell (stable sort), sets nPts, Volume,
 * the bounding box, the indenter start from IndDepth/SetupType,
 * ParticleVolume and ParticleMass, and returns N. With host_soa non-NULL
 * (after icm_allocate_arrays has set nPtsPitch) it also fills the SoA. */
int icm_load_raw_points(icy_SimParams *p, const char *path, double *host_soa, int *n_out);
/* Pinned host memory for transfer buffers (cudaMallocHost/cudaFreeHost). */
int icm_host_alloc(void **ptr, size_t bytes);
int icm_host_free(void *ptr);

#ifdef __cplusplus
} /* extern "C" */
#endif

#endif /* ICEMPM_H */
