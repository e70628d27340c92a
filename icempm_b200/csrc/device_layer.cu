// device_layer.cu -- the C ABI device layer (include/icempm.h).
//
// One icm_ctx replaces one GPU_Implementation5 (gpu_implementation5.h:40-72):
// it owns a CUDA stream, two timing events, the reference-layout particle
// SoA / grid / force bins, and -- for the fused forms -- the internal tile-
// ordered particle arrays, three grid buffers and the binning scratch.
//
// Which copy of the particle state is current is tracked explicitly:
//   ref_valid       the reference SoA on the device holds the state;
//   internal_valid  the tile-ordered arrays hold the state.
// Fused runs pack (bin + gather) from the reference SoA when needed and leave
// the internal arrays current; member-style kernels and transfers unpack
// first. Nothing here falls back to the host: every failure is a status.
#include <cuda_runtime.h>
#include <cudaTypedefs.h>  // PFN_cuTensorMapEncodeTiled (reached through the runtime, no libcuda link)
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <algorithm>
#include <type_traits>
#include <vector>

#include "../../include/icempm.h"
#include "errors.h"
#include "k_stepwise.cuh"
#include "k_tiles.cuh"

using namespace icm;

#define ICM_CUDA(call)                                                                                      \
    do {                                                                                                    \
        cudaError_t e_ = (call);                                                                            \
        if (e_ != cudaSuccess)                                                                              \
            return icm::fail(ICM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));            \
    } while (0)

#define ICM_LAUNCHED(what)                                                                                  \
    do {                                                                                                    \
        cudaError_t e_ = cudaGetLastError();                                                                \
        if (e_ != cudaSuccess) return icm::fail(ICM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e_)); \
    } while (0)

namespace {

struct TileVariant { int TX, TY; };
constexpr TileVariant kVariants[4] = {{16, 8}, {16, 16}, {32, 8}, {32, 16}};

template <class T>
int dalloc(T **p, size_t count)
{
    *p = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void **)p, count * sizeof(T));
    if (e != cudaSuccess) {
        *p = nullptr;
        return icm::fail(ICM_ERR_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    }
    return ICM_OK;
}

template <class T>
void dfree(T *&p)
{
    if (p) cudaFree((void *)p);
    p = nullptr;
}

struct Binning {
    int *key = nullptr, *count = nullptr, *cell_start = nullptr, *cursor = nullptr, *perm = nullptr;
    int *chunk = nullptr, *tile_start = nullptr, *pid = nullptr;
    int *group_slots = nullptr, *group_base = nullptr, *gchunk = nullptr;
    int *lane_cell = nullptr, *cell_lane = nullptr;  // lane order of the cells of each tile
    int *nbusy = nullptr;                            // tiles holding particles (1 int)
    size_t cap_pts = 0, cap_cells = 0, cap_tiles = 0, cap_slots = 0;
};

struct Fused {
    int form = -1;  // ICM_FORM_FP64 / ICM_FORM_FP32 held in these buffers
    size_t cap_pts = 0, cap_nodes = 0, cap_tiles = 0;
    Parts64 p64{};
    Parts32 p32{};
    // spare slot arrays for re-binning (same form), swapped with the above
    Parts64 s64{};
    Parts32 s32{};
    int *spare_pid = nullptr, *slot_key = nullptr;
    size_t spare_cap = 0;
    void *grid[3] = {nullptr, nullptr, nullptr};
    uint8_t *dirty = nullptr;  // 3 * cap_tiles
    // tile scheduling: measured cost and launch order per tile
    unsigned *cost = nullptr;
    int *order = nullptr;
    int *empties = nullptr;  // the tiles without particles, for the order's empty groups
    int cost_variant = -1, cost_ntiles = -1;  // what the costs were measured on
};

}  // namespace

struct icm_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;
    int form = ICM_FORM_FP64_STEPWISE;
    int tile_variant = 1, threads = 128;
    int rebin_interval = 100;
    // heavy tiles run as two CTAs: at most split_max tiles whose measured
    // cost exceeds split_ratio times the mean over tiles with particles
    int split_max = 128;
    double split_ratio = 1.3;

    icy_SimParams prms{};
    size_t cap_pts = 0, cap_nodes = 0, pts_pitch = 0, grid_pitch = 0;
    double *d_pts = nullptr, *d_grid = nullptr, *d_bins = nullptr;
    int *d_err = nullptr;
    double *d_hist = nullptr;
    size_t hist_cap = 0;
    int hist_n = 0;
    unsigned long long *d_redo = nullptr;
    unsigned long long *d_strays = nullptr;

    // surrogate form: device copy of the network, tolerance, {accepted, exact}
    MlpWarpNet *d_mlp = nullptr;
    float mlp_tol = 0.02f;
    unsigned long long *d_mlp_counts = nullptr;
    // harvest of crushed particles' trial states (6 floats each)
    float *d_harvest = nullptr;
    unsigned *d_harvest_n = nullptr;
    unsigned harvest_cap = 0;
    int harvest_every = 0;

    // optional per-launch timing of the fused substep kernel (kModeFull)
    bool ktime = false;
    std::vector<cudaEvent_t> kev;  // pairs
    size_t kev_used = 0;
    double ktime_ms = 0;
    long long ktime_count = 0;

    bool ref_valid = true, internal_valid = false, internal_pq = false;
    // the next fused launch may be a programmatic dependent of the kernel
    // before it: false after a kernel whose writes (launch order, re-binned
    // cells and groups) the substep reads before its griddepcontrol.wait
    bool pdl_next = false;
    int internal_variant = -1;
    int nslots = 0;
    int *h_ns = nullptr;  // pinned: the slot count and busy tiles a re-binning reads back
    int nbusy = 0;        // tiles holding particles in the current binning
    // TMA descriptors of the three grid buffers (device copy) and what they
    // were encoded for
    CUtensorMap *d_tmap = nullptr;
    TmapSet h_tmap{};  // host copy: the kernel parameter of single runs
    bool tmap_ok = false;
    void *tmap_grid[3] = {nullptr, nullptr, nullptr};
    int tmap_gx = -1, tmap_gy = -1, tmap_form = -1, tmap_variant = -1;
    Binning bin;
    Fused fz;
};

// ------------------------------------------------------------ helpers

// the internal storage of a form: the surrogate form keeps FP32 state
// the particle layout a form keeps on the device (the FP32 variants share the FP32 one)
static int storage_form(int form)
{
    return (form == ICM_FORM_FP32_SURROGATE || form == ICM_FORM_FP32_COMPENSATED) ? ICM_FORM_FP32 : form;
}

static int check_params(icm_ctx *c, const icy_SimParams *p)
{
    if (!c->d_pts) return icm::fail(ICM_ERR_STATE, "arrays are not allocated (call icm_allocate_arrays)");
    if (p->nPts < 0 || (size_t)p->nPts > c->cap_pts)
        return icm::fail(ICM_ERR_ARG, "nPts exceeds the allocated particle count");
    if (p->GridX < 4 || p->GridY < 4 || p->GridX > 32767 || p->GridY > 32767)
        return icm::fail(ICM_ERR_ARG, "GridX/GridY out of range [4, 32767]");
    if ((size_t)p->GridX * (size_t)p->GridY > c->cap_nodes)
        return icm::fail(ICM_ERR_ARG, "GridX*GridY exceeds the allocated grid");
    if (p->n_indenter_subdivisions < 1 || p->n_indenter_subdivisions > kMaxBins)
        return icm::fail(ICM_ERR_ARG, "n_indenter_subdivisions out of range [1, 256]");
    if (!(p->cellsize > 0) || !(p->InitialTimeStep > 0)) return icm::fail(ICM_ERR_ARG, "cellsize/time step not positive");
    if (p->UpdateEveryNthStep < 1) return icm::fail(ICM_ERR_ARG, "UpdateEveryNthStep < 1");
    return ICM_OK;
}

// The kernels' copy of SimParams: the caller's values with this context's
// device pointers and pitches.
static icy_SimParams kernel_params(icm_ctx *c, const icy_SimParams *p)
{
    icy_SimParams k = *p;
    k.pts_array = c->d_pts;
    k.grid_array = c->d_grid;
    k.indenter_force_accumulator = c->d_bins;
    k.nPtsPitch = c->pts_pitch;
    k.nGridPitch = c->grid_pitch;
    k.GridTotal = p->GridX * p->GridY;
    return k;
}

static Consts32 make_consts32(const icy_SimParams &P)
{
    Consts32 k{};
    k.h = (float)P.cellsize;
    k.h_inv = (float)P.cellsize_inv;
    k.dt = (float)P.InitialTimeStep;
    k.dt_h_inv = (float)(P.InitialTimeStep * P.cellsize_inv);
    k.mass = (float)P.ParticleMass;
    k.stress_c = (float)((P.InitialTimeStep * P.ParticleVolume) * P.Dp_inv);
    k.mu = (float)P.mu;
    k.kappa = (float)P.kappa;
    k.gv = (float)P.GrainVariability;
    k.ics = (float)(P.IceCompressiveStrength * 1e-6);
    k.its = (float)(P.IceTensileStrength * 1e-6);
    k.iss = (float)(P.IceShearStrength * 1e-6);
    k.four_h_inv = (float)(4.0 * P.cellsize_inv);
    k.dt_g = (float)(P.InitialTimeStep * P.Gravity);
    k.vmax = (float)(0.5 * P.cellsize / P.InitialTimeStep);
    // Wolper_Drucker_Prager (gpu_implementation5.cu:48-94): the hydrostatic
    // reset's Je_new = sqrt(-2 p_new / kappa + 1) with p_new = -p_thr
    k.p_thr = (float)P.DP_threshold_p;
    k.tan_phi = (float)P.DP_tan_phi;
    k.dp_pmax = (float)P.IceCompressiveStrength;
    k.dp_qmax = (float)P.IceShearStrength;
    {
        const double x = 2.0 * P.DP_threshold_p / P.kappa, je = std::sqrt(x + 1.0);
        k.je_new = (float)je;
        k.je_new_m1 = (float)(x / (je + 1.0));
    }
    // The box p in (-1 MPa, pmax_min / 2), q^2 < inside_q2 lies inside the
    // failure surface of every grain with residues r1 in 0..20, r2 in 0..29,
    // r3 in 0..10 (ids >= 0), by a factor of at least 4 in the terms that
    // failure_side32 compares: with a = pmax, b = -pmin, both surface
    // branches allow q^2 >= (16/9) qmax^2 ab/(a+b)^2 there, and ab/(a+b)^2
    // takes its minimum over the box of (a, b) at a corner.
    {
        const double gv = P.GrainVariability, ics = P.IceCompressiveStrength * 1e-6,
                     its = P.IceTensileStrength * 1e-6, iss = P.IceShearStrength * 1e-6;
        const double a_lo = ics * (1 + gv * 0.05 * -10), a_hi = ics * (1 + gv * 0.05 * 10);
        const double b_lo = its * (1 + gv * 0.033 * -15), b_hi = its * (1 + gv * 0.033 * 14);
        const double q_lo = iss * (1 + gv * 0.1 * -10);
        k.inside_plo = -1.0f;
        k.inside_phi = 0.0f;
        k.inside_q2 = 0.0f;
        if (a_lo > 2.0 && b_lo > 0 && q_lo > 0 && a_hi > 0 && b_hi > 0) {
            double g = 1e300;
            const double as[2] = {a_lo, a_hi}, bs[2] = {b_lo, b_hi};
            for (double a : as)
                for (double b : bs) g = std::min(g, a * b / ((a + b) * (a + b)));
            k.inside_phi = (float)(0.5 * a_lo);
            k.inside_q2 = (float)(0.25 * (16.0 / 9.0) * q_lo * q_lo * g);
        }
    }
    return k;
}

static void free_spare(icm_ctx *c)
{
    dfree(c->fz.s64.pos); dfree(c->fz.s64.F); dfree(c->fz.s64.Jp); dfree(c->fz.s64.meta);
    dfree(c->fz.s64.vel); dfree(c->fz.s64.Bp); dfree(c->fz.s64.pq);
    dfree(c->fz.s32.X); dfree(c->fz.s32.H); dfree(c->fz.s32.Jp);
    dfree(c->fz.s32.vel); dfree(c->fz.s32.Bp); dfree(c->fz.s32.pq);
    dfree(c->fz.spare_pid);
    dfree(c->fz.slot_key);
    c->fz.spare_cap = 0;
}

static void free_fused(icm_ctx *c)
{
    free_spare(c);
    dfree(c->fz.p64.pos); dfree(c->fz.p64.F); dfree(c->fz.p64.Jp); dfree(c->fz.p64.meta);
    dfree(c->fz.p64.vel); dfree(c->fz.p64.Bp); dfree(c->fz.p64.pq);
    dfree(c->fz.p32.X); dfree(c->fz.p32.H); dfree(c->fz.p32.Jp);
    dfree(c->fz.p32.vel); dfree(c->fz.p32.Bp); dfree(c->fz.p32.pq);
    for (int b = 0; b < 3; b++) { if (c->fz.grid[b]) cudaFree(c->fz.grid[b]); c->fz.grid[b] = nullptr; }
    dfree(c->fz.dirty);
    dfree(c->fz.cost); dfree(c->fz.order); dfree(c->fz.empties);
    c->fz = Fused{};
}

static void free_binning(icm_ctx *c)
{
    dfree(c->bin.key); dfree(c->bin.count); dfree(c->bin.cell_start); dfree(c->bin.cursor);
    dfree(c->bin.perm); dfree(c->bin.chunk); dfree(c->bin.tile_start); dfree(c->bin.pid);
    dfree(c->bin.group_slots); dfree(c->bin.group_base); dfree(c->bin.gchunk);
    dfree(c->bin.lane_cell); dfree(c->bin.cell_lane); dfree(c->bin.nbusy);
    c->bin = Binning{};
}

static void geometry(const icy_SimParams &P, int variant, TileGeom &g, int &ntiles)
{
    g.TX = kVariants[variant].TX;
    g.TY = kVariants[variant].TY;
    g.ntx = (P.GridX + g.TX - 1) / g.TX;
    g.nty = (P.GridY + g.TY - 1) / g.TY;
    ntiles = g.ntx * g.nty;
}

// Grid buffers, dirty flags and binning scratch of the fused forms.
static int ensure_grids(icm_ctx *c, int form, size_t npts, size_t nnodes, size_t ntiles, size_t ncells)
{
    if (c->fz.form != form || c->fz.cap_nodes < nnodes || c->fz.cap_tiles < ntiles) {
        for (int b = 0; b < 3; b++) { if (c->fz.grid[b]) cudaFree(c->fz.grid[b]); c->fz.grid[b] = nullptr; }
        dfree(c->fz.dirty);
        dfree(c->fz.cost); dfree(c->fz.order); dfree(c->fz.empties);
        c->fz.cost_variant = -1;
        c->fz.cap_nodes = nnodes;
        c->fz.cap_tiles = ntiles;
        int rc = ICM_OK;
        for (int b = 0; b < 3; b++) {
            if (form == ICM_FORM_FP64) {
                Node64 *g;
                if ((rc = dalloc(&g, nnodes))) return rc;
                c->fz.grid[b] = g;
            } else {
                float4 *g;
                if ((rc = dalloc(&g, nnodes))) return rc;
                c->fz.grid[b] = g;
            }
        }
        // cost: a tile's two halves; order: the tiles plus at most one
        // extra CTA per tile (the second halves of split tiles)
        if ((rc = dalloc(&c->fz.dirty, 3 * ntiles)) || (rc = dalloc(&c->fz.cost, 2 * ntiles)) ||
            (rc = dalloc(&c->fz.order, 2 * ntiles)) || (rc = dalloc(&c->fz.empties, ntiles)))
            return rc;
    }
    if (c->bin.cap_pts < npts || c->bin.cap_cells < ncells || c->bin.cap_tiles < ntiles) {
        int *pid = c->bin.pid;  // slot-sized, managed by ensure_slots
        size_t cap_slots = c->bin.cap_slots;
        c->bin.pid = nullptr;
        free_binning(c);
        c->bin.pid = pid;
        c->bin.cap_slots = cap_slots;
        int rc;
        size_t nchunks = (ncells + kScanChunk - 1) / kScanChunk;
        size_t ngroups = ncells / 32;
        size_t ngchunks = (ngroups + kScanChunk - 1) / kScanChunk;
        if ((rc = dalloc(&c->bin.key, npts)) || (rc = dalloc(&c->bin.perm, npts)) ||
            (rc = dalloc(&c->bin.count, ncells + 1)) || (rc = dalloc(&c->bin.cell_start, ncells + 1)) ||
            (rc = dalloc(&c->bin.cursor, ncells + 1)) || (rc = dalloc(&c->bin.chunk, nchunks + 1)) ||
            (rc = dalloc(&c->bin.tile_start, ntiles + 1)) || (rc = dalloc(&c->bin.group_slots, ngroups + 1)) ||
            (rc = dalloc(&c->bin.group_base, ngroups + 1)) || (rc = dalloc(&c->bin.gchunk, ngchunks + 1)) ||
            (rc = dalloc(&c->bin.lane_cell, ncells)) || (rc = dalloc(&c->bin.cell_lane, ncells)) ||
            (rc = dalloc(&c->bin.nbusy, 1)))
            return rc;
        c->bin.cap_pts = npts;
        c->bin.cap_cells = ncells;
        c->bin.cap_tiles = ntiles;
    }
    return ICM_OK;
}

// Slot-ordered particle arrays of one form (and the slot -> particle map).
static int ensure_slots(icm_ctx *c, int form, size_t nslots)
{
    if (c->fz.form == form && c->fz.cap_pts >= nslots && c->bin.cap_slots >= nslots) return ICM_OK;
    dfree(c->fz.p64.pos); dfree(c->fz.p64.F); dfree(c->fz.p64.Jp); dfree(c->fz.p64.meta);
    dfree(c->fz.p64.vel); dfree(c->fz.p64.Bp); dfree(c->fz.p64.pq);
    dfree(c->fz.p32.X); dfree(c->fz.p32.H); dfree(c->fz.p32.Jp);
    dfree(c->fz.p32.vel); dfree(c->fz.p32.Bp); dfree(c->fz.p32.pq);
    dfree(c->bin.pid);
    free_spare(c);
    // the same headroom as the spare set: re-binning swaps the two sets, and
    // the slot count grows as crushing packs more particles into fewer cells
    nslots += nslots / 2 + 4096;
    c->fz.form = form;
    c->fz.cap_pts = nslots;
    c->bin.cap_slots = nslots;
    int rc = ICM_OK;
    if ((rc = dalloc(&c->bin.pid, nslots))) return rc;
    if (form == ICM_FORM_FP64) {
        Parts64 &A = c->fz.p64;
        if ((rc = dalloc(&A.pos, nslots)) || (rc = dalloc(&A.F, nslots)) || (rc = dalloc(&A.Jp, nslots)) ||
            (rc = dalloc(&A.meta, nslots)) || (rc = dalloc(&A.vel, nslots)) || (rc = dalloc(&A.Bp, nslots)) ||
            (rc = dalloc(&A.pq, nslots)))
            return rc;
    } else {
        Parts32 &A = c->fz.p32;
        if ((rc = dalloc(&A.X, nslots)) || (rc = dalloc(&A.H, nslots)) ||
            (rc = dalloc(&A.Jp, nslots)) || (rc = dalloc(&A.vel, nslots)) ||
            (rc = dalloc(&A.Bp, nslots)) || (rc = dalloc(&A.pq, nslots)))
            return rc;
    }
    return ICM_OK;
}

// Exclusive scan of n ints (n + 1 outputs) with the chunked scan kernels.
static int scan_ints(icm_ctx *c, const int *in, int n, int *chunk, int *out)
{
    const int nchunks = (n + kScanChunk - 1) / kScanChunk;
    if (nchunks > kScanChunk) return icm::fail(ICM_ERR_ARG, "scan too large");
    if (n == 0) {
        ICM_CUDA(cudaMemsetAsync(out, 0, sizeof(int), c->stream));
        return ICM_OK;
    }
    // a few chunks: one block; more: the chunks' sums, then each chunk's
    // scan offset by the sums before it
    if (n <= kScanThreads * kScanSmallItems) {
        k_scan_small<<<1, kScanThreads, 0, c->stream>>>(in, n, out);
        ICM_LAUNCHED("k_scan_small");
        return ICM_OK;
    }
    k_scan_chunks<<<nchunks, kScanThreads, 0, c->stream>>>(in, n, chunk);
    ICM_LAUNCHED("k_scan_chunks");
    k_scan_apply<<<nchunks, kScanThreads, 0, c->stream>>>(in, n, chunk, out);
    ICM_LAUNCHED("k_scan_apply");
    return ICM_OK;
}

static int ensure_spare(icm_ctx *c, size_t nslots);

// Bins the reference SoA by tile and base node and gathers it into the
// internal arrays of form c->form (and makes sure the spare set that
// re-binning gathers into exists, so that no run allocates).
static int pack(icm_ctx *c, const icy_SimParams &P)
{
    TileGeom g;
    int ntiles;
    geometry(P, c->tile_variant, g, ntiles);
    const size_t ncells = (size_t)ntiles * g.TX * g.TY;
    if (ncells > (size_t)kScanChunk * kScanChunk) return icm::fail(ICM_ERR_ARG, "grid too large for the binning scan");
    int rc = ensure_grids(c, storage_form(c->form), (size_t)P.nPts, (size_t)P.GridX * P.GridY, (size_t)ntiles, ncells);
    if (rc) return rc;
    cudaStream_t s = c->stream;
    const int n = P.nPts;
    const int ngroups = (int)(ncells / 32);
    ICM_CUDA(cudaMemsetAsync(c->bin.count, 0, sizeof(int) * (ncells + 1), s));
    if (n > 0) {
        k_bin_keys<<<(n + 255) / 256, 256, 0, s>>>(P, g, c->bin.key, c->bin.count);
        ICM_LAUNCHED("k_bin_keys");
    }
    if ((rc = scan_ints(c, c->bin.count, (int)ncells, c->bin.chunk, c->bin.cell_start))) return rc;
    ICM_CUDA(cudaMemcpyAsync(c->bin.cursor, c->bin.cell_start, sizeof(int) * ncells, cudaMemcpyDeviceToDevice, s));
    if (n > 0) {
        k_bin_scatter<<<(n + 255) / 256, 256, 0, s>>>(n, c->bin.key, c->bin.cursor, c->bin.perm);
        ICM_LAUNCHED("k_bin_scatter");
    }
    k_bin_order<<<(int)((ncells + 255) / 256), 256, 0, s>>>((int)ncells, c->bin.cell_start, c->bin.perm);
    ICM_LAUNCHED("k_bin_order");
    ICM_CUDA(cudaMemsetAsync(c->bin.nbusy, 0, sizeof(int), s));
    k_lane_order<<<(ntiles + kLaneOrderWarps - 1) / kLaneOrderWarps, 32 * kLaneOrderWarps, 0, s>>>(
        ntiles, g.TX * g.TY, c->bin.cell_start, c->bin.lane_cell, c->bin.cell_lane, c->bin.group_slots,
        c->bin.tile_start, c->bin.nbusy);
    ICM_LAUNCHED("k_lane_order");
    if ((rc = scan_ints(c, c->bin.group_slots, ngroups, c->bin.gchunk, c->bin.group_base))) return rc;
    int nslots = 0, nbusy = 0;
    ICM_CUDA(cudaMemcpyAsync(&nslots, c->bin.group_base + ngroups, sizeof(int), cudaMemcpyDeviceToHost, s));
    ICM_CUDA(cudaMemcpyAsync(&nbusy, c->bin.nbusy, sizeof(int), cudaMemcpyDeviceToHost, s));
    ICM_CUDA(cudaStreamSynchronize(s));
    c->nbusy = nbusy;
    if ((rc = ensure_slots(c, storage_form(c->form), (size_t)std::max(nslots, 1)))) return rc;
    if ((rc = ensure_spare(c, (size_t)std::max(nslots, 1)))) return rc;
    ICM_CUDA(cudaMemsetAsync(c->bin.pid, 0xff, sizeof(int) * (size_t)std::max(nslots, 1), s));
    if (n > 0) {
        if (storage_form(c->form) == ICM_FORM_FP64)
            k_pack64<<<(n + 255) / 256, 256, 0, s>>>(P, c->bin.perm, c->bin.key, c->bin.cell_start,
                                                     c->bin.cell_lane, c->bin.group_base,
                                                     c->bin.pid, c->fz.p64);
        else
            k_pack32<<<(n + 255) / 256, 256, 0, s>>>(P, c->bin.perm, c->bin.key, c->bin.cell_start,
                                                     c->bin.cell_lane, c->bin.group_base,
                                                     c->bin.pid, c->fz.p32);
        ICM_LAUNCHED("k_pack");
    }
    c->nslots = nslots;
    c->internal_valid = true;
    c->internal_variant = c->tile_variant;
    c->internal_pq = false;
    return ICM_OK;
}

// Writes the internal state back into the reference SoA if it is current.
static int ensure_ref(icm_ctx *c)
{
    if (c->ref_valid) return ICM_OK;
    if (!c->internal_valid) return icm::fail(ICM_ERR_STATE, "no valid particle state on the device");
    const icy_SimParams P = kernel_params(c, &c->prms);
    const int ns = c->nslots;
    if (ns > 0 && P.nPts > 0) {
        if (c->fz.form == ICM_FORM_FP64)
            k_unpack64<<<(ns + 255) / 256, 256, 0, c->stream>>>(P, ns, c->bin.pid, c->fz.p64, c->internal_pq ? 1 : 0);
        else
            k_unpack32<<<(ns + 255) / 256, 256, 0, c->stream>>>(P, ns, c->bin.pid, c->fz.p32, c->internal_pq ? 1 : 0);
        ICM_LAUNCHED("k_unpack");
    }
    c->ref_valid = true;
    return ICM_OK;
}

static int ensure_hist(icm_ctx *c, int n)
{
    if ((size_t)n * 2 > c->hist_cap) {
        dfree(c->d_hist);
        size_t cap = std::max<size_t>(2 * (size_t)n, 1024);
        int rc = dalloc(&c->d_hist, cap);
        if (rc) return rc;
        c->hist_cap = cap;
    }
    return ICM_OK;
}

// ----------------------------------------------------- fused run dispatch

// cudaFuncSetAttribute acts on the current device, so the largest dynamic
// shared memory a kernel has been opted in to is kept per device.
constexpr int kMaxDevices = 64;
static bool need_opt_in(const size_t *opted, int device, size_t dyn)
{
    return device < 0 || device >= kMaxDevices || dyn > opted[device];
}
static void opted_in(size_t *opted, int device, size_t dyn)
{
    if (device >= 0 && device < kMaxDevices) opted[device] = dyn;
}

// Dynamic shared memory of the per-warp accumulation regions; above 48 KB
// the kernel has to opt in once.
template <class Pol, int TX, int TY, int MODE>
static int launch_one(icm_ctx *c, int ntiles, const icy_SimParams &P, const typename Pol::Consts &K,
                      const typename Pol::Parts &A, const TileRun &R)
{
    constexpr int RN = (TX + 4) * (TY + 4);
    const int nwarps = c->threads / 32;
    if (TX * TY > 32 * kMaxGroupsPerWarp * nwarps || nwarps > kMaxWarps)
        return icm::fail(ICM_ERR_ARG, "tile too large for the block size (need threads >= TX*TY/4)");
    const size_t dyn = tile_dyn_bytes<Pol, MODE>(RN, nwarps);
    static size_t opted[kMaxDevices] = {};  // static + dynamic shared memory above 48 KB needs the opt-in
    if (need_opt_in(opted, c->device, dyn)) {
        ICM_CUDA(cudaFuncSetAttribute(k_tile_substep<Pol, TX, TY, MODE>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)dyn));
        opted_in(opted, c->device, dyn);
    }
    // programmatic dependent launch: the next substep's CTAs are launched
    // while this one's last wave runs, and wait in the kernel (griddepcontrol)
    // until it has completed
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(ntiles);
    cfg.blockDim = dim3(c->threads);
    cfg.dynamicSmemBytes = dyn;
    cfg.stream = c->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = c->pdl_next ? 1 : 0;
    ICM_CUDA(cudaLaunchKernelEx(&cfg, k_tile_substep<Pol, TX, TY, MODE>, P, K, A, R, c->h_tmap));
    c->pdl_next = true;
    ICM_LAUNCHED("k_tile_substep");
    return ICM_OK;
}

template <class Pol, int TX, int TY>
static int launch_tile(icm_ctx *c, int mode, int ntiles, const icy_SimParams &P, const typename Pol::Consts &K,
                       const typename Pol::Parts &A, const TileRun &R)
{
    switch (mode) {
    case kModeP2GOnly: return launch_one<Pol, TX, TY, kModeP2GOnly>(c, ntiles, P, K, A, R);
    case kModeFull: return launch_one<Pol, TX, TY, kModeFull>(c, ntiles, P, K, A, R);
    default: return launch_one<Pol, TX, TY, kModeFinal>(c, ntiles, P, K, A, R);
    }
}

template <class Pol>
static int launch_variant(icm_ctx *c, int mode, int ntiles, const icy_SimParams &P, const typename Pol::Consts &K,
                          const typename Pol::Parts &A, const TileRun &R)
{
    switch (c->tile_variant) {
    case 0: return launch_tile<Pol, 16, 8>(c, mode, ntiles, P, K, A, R);
    case 1: return launch_tile<Pol, 16, 16>(c, mode, ntiles, P, K, A, R);
    case 2: return launch_tile<Pol, 32, 8>(c, mode, ntiles, P, K, A, R);
    default: return launch_tile<Pol, 32, 16>(c, mode, ntiles, P, K, A, R);
    }
}

// Spare arrays of nslots slots for the current form (vel/Bp are not copied by
// re-binning; the spare set gets them anyway so that a swap keeps every
// array valid in size).
static int ensure_spare(icm_ctx *c, size_t nslots)
{
    if (c->fz.spare_cap >= nslots) return ICM_OK;
    free_spare(c);
    // headroom: the slot count changes at every re-binning (it grows as
    // crushing packs more particles into fewer cells), and a reallocation
    // (cudaFree synchronises the device) costs far more than the memory
    nslots += nslots / 2 + 4096;
    int rc;
    if ((rc = dalloc(&c->fz.spare_pid, nslots)) || (rc = dalloc(&c->fz.slot_key, nslots))) return rc;
    if (c->fz.form == ICM_FORM_FP64) {
        Parts64 &A = c->fz.s64;
        if ((rc = dalloc(&A.pos, nslots)) || (rc = dalloc(&A.F, nslots)) || (rc = dalloc(&A.Jp, nslots)) ||
            (rc = dalloc(&A.meta, nslots)) || (rc = dalloc(&A.vel, nslots)) || (rc = dalloc(&A.Bp, nslots)) ||
            (rc = dalloc(&A.pq, nslots)))
            return rc;
    } else {
        Parts32 &A = c->fz.s32;
        if ((rc = dalloc(&A.X, nslots)) || (rc = dalloc(&A.H, nslots)) ||
            (rc = dalloc(&A.Jp, nslots)) || (rc = dalloc(&A.vel, nslots)) ||
            (rc = dalloc(&A.Bp, nslots)) || (rc = dalloc(&A.pq, nslots)))
            return rc;
    }
    c->fz.spare_cap = nslots;
    return ICM_OK;
}

// Re-bins the internal (slot-ordered) particle arrays by their current base
// nodes. Only valid between steady-state launches of a run. Two halves: the
// first ends with the new slot count on its way to c->h_ns, the second
// (after the caller synchronised c->stream) gathers into the new layout.
static int rebin_begin(icm_ctx *c, const icy_SimParams &P)
{
    TileGeom g;
    int ntiles;
    geometry(P, c->internal_variant, g, ntiles);
    const size_t ncells = (size_t)ntiles * g.TX * g.TY;
    const int ngroups = (int)(ncells / 32);
    const int ns_old = c->nslots;
    cudaStream_t s = c->stream;
    int rc = ensure_spare(c, (size_t)std::max(ns_old, 1));
    if (rc) return rc;
    ICM_CUDA(cudaMemsetAsync(c->bin.count, 0, sizeof(int) * (ncells + 1), s));
    const Consts32 K32 = make_consts32(P);
    const Pol64::Consts K64{0};
    if (ns_old > 0) {
        if (c->fz.form == ICM_FORM_FP64)
            k_rebin_keys<Pol64><<<(ns_old + 255) / 256, 256, 0, s>>>(P, K64, g, ns_old, c->bin.pid, c->fz.p64,
                                                                       c->fz.slot_key, c->bin.count);
        else
            k_rebin_keys<Pol32><<<(ns_old + 255) / 256, 256, 0, s>>>(P, K32, g, ns_old, c->bin.pid, c->fz.p32,
                                                                       c->fz.slot_key, c->bin.count);
        ICM_LAUNCHED("k_rebin_keys");
    }
    if ((rc = scan_ints(c, c->bin.count, (int)ncells, c->bin.chunk, c->bin.cell_start))) return rc;
    ICM_CUDA(cudaMemcpyAsync(c->bin.cursor, c->bin.cell_start, sizeof(int) * ncells, cudaMemcpyDeviceToDevice, s));
    if (ns_old > 0) {
        k_rebin_scatter<<<(ns_old + 255) / 256, 256, 0, s>>>(ns_old, c->bin.pid, c->fz.slot_key, c->bin.cursor,
                                                            c->bin.perm);
        ICM_LAUNCHED("k_rebin_scatter");
    }
    k_rebin_order<<<(int)((ncells + 255) / 256), 256, 0, s>>>((int)ncells, c->bin.cell_start, c->bin.perm, c->bin.pid);
    ICM_LAUNCHED("k_rebin_order");
    ICM_CUDA(cudaMemsetAsync(c->bin.nbusy, 0, sizeof(int), s));
    k_lane_order<<<(ntiles + kLaneOrderWarps - 1) / kLaneOrderWarps, 32 * kLaneOrderWarps, 0, s>>>(
        ntiles, g.TX * g.TY, c->bin.cell_start, c->bin.lane_cell, c->bin.cell_lane, c->bin.group_slots,
        c->bin.tile_start, c->bin.nbusy);
    ICM_LAUNCHED("k_lane_order");
    if ((rc = scan_ints(c, c->bin.group_slots, ngroups, c->bin.gchunk, c->bin.group_base))) return rc;
    if (!c->h_ns && cudaMallocHost((void **)&c->h_ns, 2 * sizeof(int)) != cudaSuccess) {
        c->h_ns = nullptr;
        return icm::fail(ICM_ERR_NOMEM, "re-binning: pinned slot count");
    }
    ICM_CUDA(cudaMemcpyAsync(c->h_ns, c->bin.group_base + ngroups, sizeof(int), cudaMemcpyDeviceToHost, s));
    ICM_CUDA(cudaMemcpyAsync(c->h_ns + 1, c->bin.nbusy, sizeof(int), cudaMemcpyDeviceToHost, s));
    return ICM_OK;
}

static int rebin_finish(icm_ctx *c, const icy_SimParams &P, bool keep_pq)
{
    TileGeom g;
    int ntiles;
    geometry(P, c->internal_variant, g, ntiles);
    const size_t ncells = (size_t)ntiles * g.TX * g.TY;
    const int ns_old = c->nslots, n = P.nPts;
    cudaStream_t s = c->stream;
    const Consts32 K32 = make_consts32(P);
    const Pol64::Consts K64{0};
    int rc;
    const int ns_new = c->h_ns[0];
    c->nbusy = c->h_ns[1];
    if ((size_t)ns_new > c->fz.spare_cap) {
        // the spare set must hold the new layout; grow it (contents of the
        // current set are untouched)
        free_spare(c);
        if ((rc = ensure_spare(c, (size_t)ns_new))) return rc;
        // slot keys were lost with the old spare set: recompute them
        ICM_CUDA(cudaMemsetAsync(c->bin.count, 0, sizeof(int) * (ncells + 1), s));
        if (c->fz.form == ICM_FORM_FP64)
            k_rebin_keys<Pol64><<<(ns_old + 255) / 256, 256, 0, s>>>(P, K64, g, ns_old, c->bin.pid, c->fz.p64,
                                                                       c->fz.slot_key, c->bin.count);
        else
            k_rebin_keys<Pol32><<<(ns_old + 255) / 256, 256, 0, s>>>(P, K32, g, ns_old, c->bin.pid, c->fz.p32,
                                                                       c->fz.slot_key, c->bin.count);
        ICM_LAUNCHED("k_rebin_keys");
    }
    ICM_CUDA(cudaMemsetAsync(c->fz.spare_pid, 0xff, sizeof(int) * (size_t)std::max(ns_new, 1), s));
    if (n > 0) {
        if (c->fz.form == ICM_FORM_FP64)
            k_rebin_gather<Parts64><<<(n + 255) / 256, 256, 0, s>>>(n, c->bin.perm, c->fz.slot_key, c->bin.cell_start,
                                                                    c->bin.cell_lane, c->bin.group_base, c->bin.pid, c->fz.spare_pid,
                                                                    c->fz.p64, c->fz.s64, keep_pq ? 1 : 0);
        else
            k_rebin_gather<Parts32><<<(n + 255) / 256, 256, 0, s>>>(n, c->bin.perm, c->fz.slot_key, c->bin.cell_start,
                                                                    c->bin.cell_lane, c->bin.group_base, c->bin.pid, c->fz.spare_pid,
                                                                    c->fz.p32, c->fz.s32, keep_pq ? 1 : 0);
        ICM_LAUNCHED("k_rebin_gather");
    }
    std::swap(c->fz.p64, c->fz.s64);
    std::swap(c->fz.p32, c->fz.s32);
    std::swap(c->bin.pid, c->fz.spare_pid);
    std::swap(c->fz.cap_pts, c->fz.spare_cap);
    c->bin.cap_slots = c->fz.cap_pts;
    c->nslots = ns_new;
    return ICM_OK;
}

static int rebin_internal(icm_ctx *c, const icy_SimParams &P, bool keep_pq)
{
    int rc = rebin_begin(c, P);
    if (rc) return rc;
    ICM_CUDA(cudaStreamSynchronize(c->stream));
    c->pdl_next = false;  // the substep reads cells and groups before its dependency wait
    return rebin_finish(c, P, keep_pq);
}

// TMA descriptors of the grid buffers for the node-region copies of the
// fused kernel: 2D maps of {4 GridX, GridY} floats (doubles in the FP64
// form) with a box of {4 (TX+4), TY+4}. The runtime hands out the driver's
// encoder; where it is missing or refuses, the kernel keeps its plain loads.
static PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
        else
            cudaGetLastError();
    }
    return fn;
}

static int ensure_tmaps(icm_ctx *c, const icy_SimParams &P)
{
    const int form = storage_form(c->form);
    if (c->tmap_form == form && c->tmap_variant == c->tile_variant && c->tmap_gx == P.GridX && c->tmap_gy == P.GridY &&
        c->tmap_grid[0] == c->fz.grid[0] && c->tmap_grid[1] == c->fz.grid[1] && c->tmap_grid[2] == c->fz.grid[2])
        return ICM_OK;
    c->tmap_ok = false;
    c->tmap_form = form;
    c->tmap_variant = c->tile_variant;
    c->tmap_gx = P.GridX;
    c->tmap_gy = P.GridY;
    for (int b = 0; b < 3; b++) c->tmap_grid[b] = c->fz.grid[b];
    PFN_cuTensorMapEncodeTiled_v12000 enc = tmap_encoder();
    if (!enc) return ICM_OK;
    if (!c->d_tmap) {
        if (cudaMalloc((void **)&c->d_tmap, 3 * sizeof(CUtensorMap)) != cudaSuccess) {
            c->d_tmap = nullptr;
            return icm::fail(ICM_ERR_NOMEM, "tensor maps");
        }
    }
    const TileVariant tv = kVariants[c->tile_variant];
    const size_t elem = (form == ICM_FORM_FP64) ? sizeof(double) : sizeof(float);
    CUtensorMap h[3];
    for (int b = 0; b < 3; b++) {
        const cuuint64_t dims[2] = {4 * (cuuint64_t)P.GridX, (cuuint64_t)P.GridY};
        const cuuint64_t strides[1] = {4 * elem * (cuuint64_t)P.GridX};
        const cuuint32_t box[2] = {4 * (cuuint32_t)(tv.TX + 4), (cuuint32_t)(tv.TY + 4)};
        const cuuint32_t es[2] = {1, 1};
        const CUresult r = enc(&h[b], form == ICM_FORM_FP64 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                               2, c->fz.grid[b], dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return ICM_OK;
    }
    ICM_CUDA(cudaMemcpyAsync(c->d_tmap, h, sizeof(h), cudaMemcpyHostToDevice, c->stream));
    ICM_CUDA(cudaStreamSynchronize(c->stream));  // h goes out of scope
    for (int b = 0; b < 3; b++) c->h_tmap.m[b] = h[b];
    c->tmap_ok = true;
    return ICM_OK;
}

// Tile order for the next launches: by the costs measured on this tile
// geometry, the heaviest tiles split over two CTAs; or the identity (null)
// while there are no costs. nlaunch: the grid of the fused launches.
static int tile_order(icm_ctx *c, int ntiles, const int *&order, int &nlaunch)
{
    order = nullptr;
    nlaunch = ntiles;
    if (c->fz.cost_variant != c->tile_variant || c->fz.cost_ntiles != ntiles) {
        ICM_CUDA(cudaMemsetAsync(c->fz.cost, 0, 2 * sizeof(unsigned) * (size_t)ntiles, c->stream));
        c->fz.cost_variant = c->tile_variant;
        c->fz.cost_ntiles = ntiles;
        return ICM_OK;
    }
    if (ntiles > kMaxOrderTiles) return ICM_OK;
    const int max_split = std::min(std::max(c->split_max, 0), ntiles);
    static size_t opted[kMaxDevices] = {};  // 2 ints per tile: above 48 KB from 6,144 tiles
    const size_t order_smem = 2 * sizeof(int) * kMaxOrderTiles;
    if (need_opt_in(opted, c->device, order_smem)) {
        ICM_CUDA(cudaFuncSetAttribute(k_tile_order, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)order_smem));
        opted_in(opted, c->device, order_smem);
    }
    k_tile_order<<<1, kOrderThreads, 2 * sizeof(int) * (size_t)ntiles, c->stream>>>(
        ntiles, c->fz.cost, c->bin.tile_start, max_split, (float)c->split_ratio, c->fz.order, c->fz.empties);
    ICM_LAUNCHED("k_tile_order");
    c->pdl_next = false;  // the substep reads the order before its dependency wait
    order = c->fz.order;
    // the busy tiles, the second halves of at most max_split split tiles and
    // the groups of tiles without particles (entries past the used ones are -1)
    const int nbusy = std::min(std::max(c->nbusy, 0), ntiles);
    nlaunch = nbusy + max_split + (ntiles - nbusy + kEmptyPerCta - 1) / kEmptyPerCta;
    return ICM_OK;
}

static int run_fused(icm_ctx *c, icy_SimParams *p, int n)
{
    icy_SimParams P = kernel_params(c, p);
    if (c->form == ICM_FORM_FP32_SURROGATE && !c->d_mlp)
        return icm::fail(ICM_ERR_STATE, "surrogate form without a network (icm_set_surrogate)");
    if (c->form == ICM_FORM_FP32_SURROGATE && c->threads > 32 * Pol32S::kWarps)
        return icm::fail(ICM_ERR_ARG, "surrogate form: at most 128 threads per block");
    if (!c->internal_valid || c->fz.form != storage_form(c->form) || c->internal_variant != c->tile_variant) {
        int rc = ensure_ref(c);
        if (rc) return rc;
        if ((rc = pack(c, P))) return rc;
    }
    TileGeom g;
    int ntiles;
    geometry(P, c->tile_variant, g, ntiles);
    const size_t nnodes = (size_t)P.GridX * P.GridY;
    const size_t node_bytes = (storage_form(c->form) == ICM_FORM_FP64) ? sizeof(Node64) : sizeof(float4);
    cudaStream_t s = c->stream;
    c->pdl_next = false;  // packing or an earlier run's kernels precede the prologue
    for (int b = 0; b < 3; b++) ICM_CUDA(cudaMemsetAsync(c->fz.grid[b], 0, node_bytes * nnodes, s));
    ICM_CUDA(cudaMemsetAsync(c->fz.dirty, 0, 3 * (size_t)ntiles, s));
    int rc = ensure_hist(c, n);
    if (rc) return rc;
    ICM_CUDA(cudaMemsetAsync(c->d_hist, 0, sizeof(double) * 2 * (size_t)n, s));
    c->hist_n = n;

    TileRun R{};
    R.ntx = g.ntx;
    R.nty = g.nty;
    R.tile_start = c->bin.tile_start;
    for (int b = 0; b < 3; b++) {
        R.dirty[b] = c->fz.dirty + (size_t)b * ntiles;
        R.grid[b] = c->fz.grid[b];
    }
    R.bins = c->d_bins;
    R.err = c->d_err;
    R.fp64_redo = c->d_redo;
    R.cell_start = c->bin.cell_start;
    R.lane_cell = c->bin.lane_cell;
    R.group_base = c->bin.group_base;
    R.strays = c->d_strays;
    R.ind_y = p->indenter_y;
    R.cost = c->fz.cost;
    int nlaunch = ntiles;
    if ((rc = tile_order(c, ntiles, R.order, nlaunch))) return rc;
    R.empties = c->fz.empties;
    R.nempty = ntiles - std::min(std::max(c->nbusy, 0), ntiles);
    if ((rc = ensure_tmaps(c, P))) return rc;
    R.tmap = c->tmap_ok ? c->d_tmap : nullptr;

    Consts32 K32 = make_consts32(P);
    K32.mlp = c->d_mlp;
    K32.mlp_tol = c->mlp_tol;
    K32.mlp_counts = c->d_mlp_counts;
    bool harvest_now = false;  // this launch appends crushed particles' trial states
    const Pol64::Consts K64{0};
    auto launch = [&](int mode) -> int {
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (c->ktime && mode == kModeFull) {
            if (c->kev_used + 2 > c->kev.size()) {
                for (int k = 0; k < 64; k++) {
                    cudaEvent_t e;
                    if (cudaEventCreate(&e) != cudaSuccess) return icm::fail(ICM_ERR_CUDA, "cudaEventCreate");
                    c->kev.push_back(e);
                }
            }
            e0 = c->kev[c->kev_used++];
            e1 = c->kev[c->kev_used++];
            ICM_CUDA(cudaEventRecord(e0, c->stream));
        }
        int r;
        if (c->form == ICM_FORM_FP64) {
            r = launch_variant<Pol64>(c, mode, nlaunch, P, K64, c->fz.p64, R);
        } else {
            Consts32 K = K32;
            if (c->d_harvest && harvest_now) {
                K.harvest = c->d_harvest;
                K.harvest_n = c->d_harvest_n;
                K.harvest_cap = c->harvest_cap;
            }
            r = (c->form == ICM_FORM_FP32_SURROGATE)     ? launch_variant<Pol32S>(c, mode, nlaunch, P, K, c->fz.p32, R)
                : (c->form == ICM_FORM_FP32_COMPENSATED) ? launch_variant<Pol32C>(c, mode, nlaunch, P, K, c->fz.p32, R)
                                                         : launch_variant<Pol32>(c, mode, nlaunch, P, K, c->fz.p32, R);
        }
        if (e1) ICM_CUDA(cudaEventRecord(e1, c->stream));
        return r;
    };
    // prologue: P2G of the current state into G[0]
    R.bufA = 0; R.bufB = 0; R.bufC = 0;
    R.force_slot = nullptr;
    R.record_pq = 0;
    R.ind_x = p->indenter_x;
    if ((rc = launch(kModeP2GOnly))) return rc;
    double t = p->SimulationTime;
    bool any_pq = false;
    for (int k = 1; k <= n; k++) {
        t += p->InitialTimeStep;
        p->indenter_x = p->indenter_x_initial + t * p->IndVelocity;
        const int sidx = k - 1;
        R.bufA = sidx % 3;
        R.bufB = (sidx + 1) % 3;
        R.bufC = (sidx + 2) % 3;
        R.ind_x = p->indenter_x;
        R.force_slot = c->d_hist + 2 * (size_t)sidx;
        R.record_pq = ((p->SimulationStep + k) % p->UpdateEveryNthStep == 0) ? 1 : 0;
        any_pq |= R.record_pq != 0;
        harvest_now = c->harvest_every > 0 && (p->SimulationStep + k) % c->harvest_every == 0;
        if ((rc = launch(k < n ? kModeFull : kModeFinal))) return rc;
        if (k < n && c->rebin_interval > 0 && k % c->rebin_interval == 0) {
            if ((rc = rebin_internal(c, P, c->internal_pq || any_pq))) return rc;
            R.group_base = c->bin.group_base;
            if ((rc = tile_order(c, ntiles, R.order, nlaunch))) return rc;
            R.nempty = ntiles - std::min(std::max(c->nbusy, 0), ntiles);
        }
    }
    p->SimulationStep += n;
    p->SimulationTime = t;
    c->internal_valid = true;
    c->ref_valid = false;
    c->internal_pq = c->internal_pq || any_pq;
    return ICM_OK;
}

static int run_stepwise(icm_ctx *c, icy_SimParams *p, int n)
{
    int rc = ensure_ref(c);
    if (rc) return rc;
    if ((rc = ensure_hist(c, n))) return rc;
    cudaStream_t s = c->stream;
    ICM_CUDA(cudaMemsetAsync(c->d_hist, 0, sizeof(double) * 2 * (size_t)n, s));
    c->hist_n = n;
    double t = p->SimulationTime;
    for (int k = 1; k <= n; k++) {
        t += p->InitialTimeStep;
        p->indenter_x = p->indenter_x_initial + t * p->IndVelocity;
        icy_SimParams P = kernel_params(c, p);
        ICM_CUDA(cudaMemsetAsync(c->d_grid, 0, sizeof(double) * c->grid_pitch * ICM_N_GRID_ARRAYS, s));
        const int tp = P.tpb_P2G > 0 ? P.tpb_P2G : 256, tu = P.tpb_Upd > 0 ? P.tpb_Upd : 512;
        const int tg = P.tpb_G2P > 0 ? P.tpb_G2P : 128;
        if (P.nPts > 0) {
            k_p2g_ref64<<<(P.nPts + tp - 1) / tp, tp, 0, s>>>(P, c->d_err);
            ICM_LAUNCHED("cuda_p2g");
        }
        k_update_ref64<<<(P.GridTotal + tu - 1) / tu, tu, 0, s>>>(P, p->indenter_x, p->indenter_y,
                                                                  c->d_hist + 2 * (size_t)(k - 1));
        ICM_LAUNCHED("cuda_update_nodes");
        if (P.nPts > 0) {
            k_g2p_ref64<<<(P.nPts + tg - 1) / tg, tg, 0, s>>>(P, (p->SimulationStep + k) % p->UpdateEveryNthStep == 0);
            ICM_LAUNCHED("cuda_g2p");
        }
    }
    p->SimulationStep += n;
    p->SimulationTime = t;
    c->internal_valid = false;
    c->ref_valid = true;
    return ICM_OK;
}

// ------------------------------------------------------------------- ABI

extern "C" int icm_create(icm_ctx **out, int device)
{
    if (!out) return icm::fail(ICM_ERR_ARG, "icm_create: null out");
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0)
        return icm::fail(ICM_ERR_NODEVICE, std::string("No avaialble CUDA devices: ") + cudaGetErrorString(e));
    if (device < 0 || device >= count) return icm::fail(ICM_ERR_ARG, "icm_create: device index out of range");
    ICM_CUDA(cudaSetDevice(device));
    icm_ctx *c = new icm_ctx();
    c->device = device;
    if (cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreate(&c->ev_start) != cudaSuccess || cudaEventCreate(&c->ev_stop) != cudaSuccess ||
        cudaMalloc((void **)&c->d_err, sizeof(int)) != cudaSuccess ||
        cudaMalloc((void **)&c->d_redo, sizeof(unsigned long long)) != cudaSuccess ||
        cudaMalloc((void **)&c->d_strays, sizeof(unsigned long long)) != cudaSuccess) {
        icm_destroy(c);
        return icm::fail(ICM_ERR_CUDA, "icm_create: stream/event/allocation failed");
    }
    cudaMemset(c->d_err, 0, sizeof(int));
    cudaMemset(c->d_redo, 0, sizeof(unsigned long long));
    cudaMemset(c->d_strays, 0, sizeof(unsigned long long));
    *out = c;
    return ICM_OK;
}

extern "C" int icm_destroy(icm_ctx *c)
{
    if (!c) return ICM_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    free_fused(c);
    free_binning(c);
    dfree(c->d_pts); dfree(c->d_grid); dfree(c->d_bins); dfree(c->d_err); dfree(c->d_hist); dfree(c->d_redo); dfree(c->d_strays);
    dfree(c->d_mlp); dfree(c->d_mlp_counts); dfree(c->d_harvest); dfree(c->d_harvest_n);
    if (c->h_ns) cudaFreeHost(c->h_ns);
    if (c->d_tmap) cudaFree(c->d_tmap);
    for (cudaEvent_t e : c->kev) cudaEventDestroy(e);
    if (c->ev_start) cudaEventDestroy(c->ev_start);
    if (c->ev_stop) cudaEventDestroy(c->ev_stop);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return ICM_OK;
}

extern "C" int icm_set_form(icm_ctx *c, int form)
{
    if (!c) return icm::fail(ICM_ERR_ARG, "null context");
    if (form < ICM_FORM_FP64_STEPWISE || form > ICM_FORM_FP32_COMPENSATED) return icm::fail(ICM_ERR_ARG, "unknown form");
    if (form == c->form) return ICM_OK;
    if (c->d_pts) {
        int rc = ensure_ref(c);
        if (rc) return rc;
    }
    c->internal_valid = false;
    c->form = form;
    return ICM_OK;
}

extern "C" int icm_get_form(icm_ctx *c) { return c ? c->form : -1; }

extern "C" int icm_set_tile(icm_ctx *c, int variant, int threads)
{
    if (!c) return icm::fail(ICM_ERR_ARG, "null context");
    if (variant < 0 || variant > 3) return icm::fail(ICM_ERR_ARG, "tile variant must be 0..3");
    if (threads < 32 || threads > 256 || threads % 32) return icm::fail(ICM_ERR_ARG, "threads must be 32..256, multiple of 32");
    if (variant != c->tile_variant && c->d_pts) {
        int rc = ensure_ref(c);
        if (rc) return rc;
        c->internal_valid = false;
    }
    c->tile_variant = variant;
    c->threads = threads;
    return ICM_OK;
}

extern "C" int icm_set_rebin_interval(icm_ctx *c, int substeps)
{
    if (!c) return icm::fail(ICM_ERR_ARG, "null context");
    if (substeps < 0) return icm::fail(ICM_ERR_ARG, "re-binning interval must be >= 0");
    c->rebin_interval = substeps;
    return ICM_OK;
}

extern "C" int icm_set_tile_split(icm_ctx *c, int max_tiles, double ratio)
{
    if (!c) return icm::fail(ICM_ERR_ARG, "null context");
    if (max_tiles < 0 || !(ratio >= 0)) return icm::fail(ICM_ERR_ARG, "icm_set_tile_split: max_tiles >= 0, ratio >= 0");
    c->split_max = max_tiles;
    c->split_ratio = ratio;
    return ICM_OK;
}

extern "C" int icm_get_tile(icm_ctx *c, int *variant, int *threads)
{
    if (!c) return icm::fail(ICM_ERR_ARG, "null context");
    if (variant) *variant = c->tile_variant;
    if (threads) *threads = c->threads;
    return ICM_OK;
}

extern "C" int icm_allocate_arrays(icm_ctx *c, icy_SimParams *p, size_t n_grid_nodes, size_t n_points)
{
    if (!c || !p) return icm::fail(ICM_ERR_ARG, "null argument");
    if (n_points > 0x7fffffffULL || n_grid_nodes > 0x7fffffffULL) return icm::fail(ICM_ERR_ARG, "sizes too large");
    ICM_CUDA(cudaSetDevice(c->device));
    ICM_CUDA(cudaStreamSynchronize(c->stream));
    dfree(c->d_pts);
    dfree(c->d_grid);
    dfree(c->d_bins);
    free_fused(c);
    free_binning(c);
    c->pts_pitch = icm_pitch_elems(n_points);
    c->grid_pitch = icm_pitch_elems(n_grid_nodes);
    int rc;
    if ((rc = dalloc(&c->d_pts, c->pts_pitch * ICM_N_PTS_ARRAYS))) return rc;
    if ((rc = dalloc(&c->d_grid, c->grid_pitch * ICM_N_GRID_ARRAYS))) return rc;
    if ((rc = dalloc(&c->d_bins, (size_t)2 * kMaxBins))) return rc;
    ICM_CUDA(cudaMemset(c->d_pts, 0, sizeof(double) * c->pts_pitch * ICM_N_PTS_ARRAYS));
    ICM_CUDA(cudaMemset(c->d_grid, 0, sizeof(double) * c->grid_pitch * ICM_N_GRID_ARRAYS));
    ICM_CUDA(cudaMemset(c->d_bins, 0, sizeof(double) * 2 * kMaxBins));
    ICM_CUDA(cudaMemset(c->d_err, 0, sizeof(int)));
    c->cap_pts = n_points;
    c->cap_nodes = n_grid_nodes;
    p->pts_array = c->d_pts;
    p->grid_array = c->d_grid;
    p->indenter_force_accumulator = c->d_bins;
    p->nPtsPitch = c->pts_pitch;
    p->nGridPitch = c->grid_pitch;
    c->prms = *p;
    c->ref_valid = true;
    c->internal_valid = false;
    return ICM_OK;
}

extern "C" int icm_update_constants(icm_ctx *c, const icy_SimParams *p, int error_code)
{
    if (!c || !p) return icm::fail(ICM_ERR_ARG, "null argument");
    int rc = check_params(c, p);
    if (rc) return rc;
    ICM_CUDA(cudaMemcpyAsync(c->d_err, &error_code, sizeof(int), cudaMemcpyHostToDevice, c->stream));
    ICM_CUDA(cudaStreamSynchronize(c->stream));
    c->prms = *p;
    return ICM_OK;
}

extern "C" int icm_transfer_points_to_device(icm_ctx *c, const double *host_soa)
{
    if (!c || !host_soa) return icm::fail(ICM_ERR_ARG, "null argument");
    if (!c->d_pts) return icm::fail(ICM_ERR_STATE, "arrays are not allocated");
    ICM_CUDA(cudaMemcpyAsync(c->d_pts, host_soa, sizeof(double) * c->pts_pitch * ICM_N_PTS_ARRAYS,
                             cudaMemcpyHostToDevice, c->stream));
    ICM_CUDA(cudaStreamSynchronize(c->stream));
    c->ref_valid = true;
    c->internal_valid = false;
    return ICM_OK;
}

extern "C" int icm_reset_grid(icm_ctx *c)
{
    if (!c || !c->d_grid) return icm::fail(ICM_ERR_STATE, "arrays are not allocated");
    ICM_CUDA(cudaMemsetAsync(c->d_grid, 0, sizeof(double) * c->grid_pitch * ICM_N_GRID_ARRAYS, c->stream));
    return ICM_OK;
}

extern "C" int icm_reset_indenter_force_accumulator(icm_ctx *c)
{
    if (!c || !c->d_bins) return icm::fail(ICM_ERR_STATE, "arrays are not allocated");
    ICM_CUDA(cudaMemsetAsync(c->d_bins, 0, sizeof(double) * 2 * kMaxBins, c->stream));
    return ICM_OK;
}

extern "C" int icm_p2g(icm_ctx *c)
{
    if (!c) return icm::fail(ICM_ERR_ARG, "null context");
    int rc = check_params(c, &c->prms);
    if (rc || (rc = ensure_ref(c))) return rc;
    icy_SimParams P = kernel_params(c, &c->prms);
    int tpb = P.tpb_P2G > 0 ? P.tpb_P2G : 256;
    if (P.nPts > 0) {
        k_p2g_ref64<<<(P.nPts + tpb - 1) / tpb, tpb, 0, c->stream>>>(P, c->d_err);
        ICM_LAUNCHED("cuda_p2g");
    }
    return ICM_OK;
}

extern "C" int icm_update_nodes(icm_ctx *c, double indenter_x, double indenter_y)
{
    if (!c) return icm::fail(ICM_ERR_ARG, "null context");
    int rc = check_params(c, &c->prms);
    if (rc) return rc;
    icy_SimParams P = kernel_params(c, &c->prms);
    int tpb = P.tpb_Upd > 0 ? P.tpb_Upd : 512;
    k_update_ref64<<<(P.GridTotal + tpb - 1) / tpb, tpb, 0, c->stream>>>(P, indenter_x, indenter_y, nullptr);
    ICM_LAUNCHED("cuda_update_nodes");
    return ICM_OK;
}

extern "C" int icm_g2p(icm_ctx *c, int record_pq)
{
    if (!c) return icm::fail(ICM_ERR_ARG, "null context");
    int rc = check_params(c, &c->prms);
    if (rc || (rc = ensure_ref(c))) return rc;
    icy_SimParams P = kernel_params(c, &c->prms);
    int tpb = P.tpb_G2P > 0 ? P.tpb_G2P : 128;
    if (P.nPts > 0) {
        k_g2p_ref64<<<(P.nPts + tpb - 1) / tpb, tpb, 0, c->stream>>>(P, record_pq ? 1 : 0);
        ICM_LAUNCHED("cuda_g2p");
    }
    c->internal_valid = false;
    return ICM_OK;
}

extern "C" int icm_transfer_from_device(icm_ctx *c, double *host_soa, double *host_bins, int *error_code,
                                        icm_host_fn cb, void *user)
{
    if (!c) return icm::fail(ICM_ERR_ARG, "null context");
    if (!c->d_pts) return icm::fail(ICM_ERR_STATE, "arrays are not allocated");
    int rc = ensure_ref(c);
    if (rc) return rc;
    cudaStream_t s = c->stream;
    if (host_soa)
        ICM_CUDA(cudaMemcpyAsync(host_soa, c->d_pts, sizeof(double) * c->pts_pitch * ICM_N_PTS_ARRAYS,
                                 cudaMemcpyDeviceToHost, s));
    if (host_bins)
        ICM_CUDA(cudaMemcpyAsync(host_bins, c->d_bins, sizeof(double) * 2 * c->prms.n_indenter_subdivisions,
                                 cudaMemcpyDeviceToHost, s));
    if (error_code) ICM_CUDA(cudaMemcpyAsync(error_code, c->d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    if (cb) ICM_CUDA(cudaLaunchHostFunc(s, (cudaHostFn_t)cb, user));
    return ICM_OK;
}

extern "C" int icm_transfer_grid_to_device(icm_ctx *c, const double *host_grid)
{
    if (!c || !host_grid) return icm::fail(ICM_ERR_ARG, "null argument");
    if (!c->d_grid) return icm::fail(ICM_ERR_STATE, "arrays are not allocated");
    ICM_CUDA(cudaMemcpyAsync(c->d_grid, host_grid, sizeof(double) * c->grid_pitch * ICM_N_GRID_ARRAYS,
                             cudaMemcpyHostToDevice, c->stream));
    ICM_CUDA(cudaStreamSynchronize(c->stream));
    return ICM_OK;
}

extern "C" int icm_transfer_grid_from_device(icm_ctx *c, double *host_grid)
{
    if (!c || !host_grid) return icm::fail(ICM_ERR_ARG, "null argument");
    if (!c->d_grid) return icm::fail(ICM_ERR_STATE, "arrays are not allocated");
    ICM_CUDA(cudaMemcpyAsync(host_grid, c->d_grid, sizeof(double) * c->grid_pitch * ICM_N_GRID_ARRAYS,
                             cudaMemcpyDeviceToHost, c->stream));
    ICM_CUDA(cudaStreamSynchronize(c->stream));
    return ICM_OK;
}

extern "C" int icm_synchronize(icm_ctx *c)
{
    if (!c) return ICM_OK;
    ICM_CUDA(cudaStreamSynchronize(c->stream));
    return ICM_OK;
}

extern "C" int icm_run_substeps(icm_ctx *c, icy_SimParams *p, int n)
{
    if (!c || !p) return icm::fail(ICM_ERR_ARG, "null argument");
    if (n < 0) return icm::fail(ICM_ERR_ARG, "negative substep count");
    int rc = check_params(c, p);
    if (rc) return rc;
    c->prms = *p;
    if (n == 0) return ICM_OK;
    rc = (c->form == ICM_FORM_FP64_STEPWISE) ? run_stepwise(c, p, n) : run_fused(c, p, n);
    c->prms = *p;
    return rc;
}

extern "C" int icm_force_history(icm_ctx *c, double *host_out, int n)
{
    if (!c || !host_out) return icm::fail(ICM_ERR_ARG, "null argument");
    if (n < 0 || n > c->hist_n) return icm::fail(ICM_ERR_ARG, "history shorter than requested");
    if (n == 0) return ICM_OK;
    ICM_CUDA(cudaMemcpyAsync(host_out, c->d_hist, sizeof(double) * 2 * (size_t)n, cudaMemcpyDeviceToHost, c->stream));
    ICM_CUDA(cudaStreamSynchronize(c->stream));
    return ICM_OK;
}

extern "C" int icm_fp64_redo_count(icm_ctx *c, unsigned long long *out)
{
    if (!c || !out) return icm::fail(ICM_ERR_ARG, "null argument");
    ICM_CUDA(cudaMemcpyAsync(out, c->d_redo, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
    ICM_CUDA(cudaStreamSynchronize(c->stream));
    return ICM_OK;
}

extern "C" int icm_stray_count(icm_ctx *c, unsigned long long *out)
{
    if (!c || !out) return icm::fail(ICM_ERR_ARG, "null argument");
    ICM_CUDA(cudaMemcpyAsync(out, c->d_strays, sizeof(unsigned long long), cudaMemcpyDeviceToHost, c->stream));
    ICM_CUDA(cudaStreamSynchronize(c->stream));
    return ICM_OK;
}

extern "C" int icm_record_start(icm_ctx *c)
{
    if (!c) return icm::fail(ICM_ERR_ARG, "null context");
    ICM_CUDA(cudaEventRecord(c->ev_start, c->stream));
    return ICM_OK;
}

extern "C" int icm_record_stop(icm_ctx *c)
{
    if (!c) return icm::fail(ICM_ERR_ARG, "null context");
    ICM_CUDA(cudaEventRecord(c->ev_stop, c->stream));
    return ICM_OK;
}

extern "C" int icm_cycle_events(icm_ctx *c, void **start, void **stop)
{
    if (!c || !start || !stop) return icm::fail(ICM_ERR_ARG, "icm_cycle_events: null argument");
    *start = (void *)c->ev_start;
    *stop = (void *)c->ev_stop;
    return ICM_OK;
}

extern "C" int icm_elapsed_ms(icm_ctx *c, float *ms)
{
    if (!c || !ms) return icm::fail(ICM_ERR_ARG, "null argument");
    ICM_CUDA(cudaEventSynchronize(c->ev_stop));
    ICM_CUDA(cudaEventElapsedTime(ms, c->ev_start, c->ev_stop));
    return ICM_OK;
}

// Accumulates the recorded launch pairs into ktime_ms (synchronises).
static int harvest_ktime(icm_ctx *c)
{
    if (c->kev_used == 0) return ICM_OK;
    ICM_CUDA(cudaStreamSynchronize(c->stream));
    for (size_t k = 0; k + 1 < c->kev_used; k += 2) {
        float ms = 0;
        ICM_CUDA(cudaEventElapsedTime(&ms, c->kev[k], c->kev[k + 1]));
        c->ktime_ms += ms;
        c->ktime_count++;
    }
    c->kev_used = 0;
    return ICM_OK;
}

extern "C" int icm_kernel_timing(icm_ctx *c, int enable)
{
    if (!c) return icm::fail(ICM_ERR_ARG, "null context");
    int rc = harvest_ktime(c);
    if (rc) return rc;
    c->ktime = enable != 0;
    c->ktime_ms = 0;
    c->ktime_count = 0;
    return ICM_OK;
}

extern "C" int icm_kernel_time(icm_ctx *c, double *total_ms, long long *launches)
{
    if (!c || !total_ms || !launches) return icm::fail(ICM_ERR_ARG, "null argument");
    int rc = harvest_ktime(c);
    if (rc) return rc;
    *total_ms = c->ktime_ms;
    *launches = c->ktime_count;
    return ICM_OK;
}

extern "C" void *icm_stream(icm_ctx *c) { return c ? (void *)c->stream : nullptr; }

// ------------------------------------------------------------ ensembles

struct icm_ensemble {
    int device = 0;
    cudaStream_t stream = nullptr;
    int form = ICM_FORM_FP32, variant = 1, threads = 128, rebin_interval = 200;
    bool graphs = true;
    std::vector<icm_ctx *> cases;
    void *d_cases = nullptr;
    size_t cases_bytes = 0;
    int *d_tile_case = nullptr, *d_tile_local = nullptr, *d_nactive = nullptr, *d_seg_base = nullptr;
    size_t tiles_cap = 0;
    int nactive = 0;
    double *d_ind_x = nullptr;
    size_t ind_x_cap = 0;
    uint8_t *d_active = nullptr;  // every case's tile mask, concatenated
    size_t active_cap = 0;
    std::vector<size_t> active_off;
    struct Seg {
        cudaGraphExec_t exec;
        int len, grid;
    };
    std::vector<Seg> graphs_by_len;  // captured segments (at most kEnsGraphs lengths)
    std::vector<cudaEvent_t> events;  // one per case, plus one for the ensemble stream
    unsigned char *h_stage = nullptr;  // pinned: every case's tile starts, costs and dirty flags
    size_t stage_cap = 0;
    // heavy tiles split over two CTAs, as icm_set_tile_split; off by default:
    // the launch list of many cases has work enough that no single tile sets
    // its length (64 cases: 0.520 ms per substep without, 0.528 with)
    int split_max = 0;
    double split_ratio = 1.3;
};

namespace {

// a captured graph holds the descriptor and active-tile pointers: drop it
// when they are reallocated (after cudaFree's implicit synchronisation)
void ens_drop_graph(icm_ensemble *e)
{
    for (auto &g : e->graphs_by_len) cudaGraphExecDestroy(g.exec);
    e->graphs_by_len.clear();
}

constexpr int kEnsGraphs = 4;

template <class Pol, int TX, int TY, int MODE>
int ens_launch_one(icm_ensemble *e, int grid, const void *d_cases, const EnsLaunch &L)
{
    // the first launch of a segment, the prologue and the final launch follow
    // k_set_int or the descriptor upload, whose writes the kernel reads before
    // its dependency wait: they are ordinary stream-ordered launches
    const bool pdl = MODE == kModeFull && L.j > 0;
    constexpr int RN = (TX + 4) * (TY + 4);
    const int nwarps = e->threads / 32;
    const size_t dyn = tile_dyn_bytes<Pol, MODE>(RN, nwarps);
    static size_t opted[kMaxDevices] = {};
    if (need_opt_in(opted, e->device, dyn)) {
        ICM_CUDA(cudaFuncSetAttribute(k_tile_substep_ens<Pol, TX, TY, MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)dyn));
        opted_in(opted, e->device, dyn);
    }
    if (grid < 1) return ICM_OK;
    // a programmatic dependent of the previous launch, as single runs are
    // (inside a captured segment this becomes a programmatic graph edge)
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(e->threads);
    cfg.dynamicSmemBytes = dyn;
    cfg.stream = e->stream;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    ICM_CUDA(cudaLaunchKernelEx(&cfg, k_tile_substep_ens<Pol, TX, TY, MODE>, static_cast<const EnsCase<Pol> *>(d_cases),
                                L));
    ICM_LAUNCHED("k_tile_substep_ens");
    return ICM_OK;
}

template <class Pol, int TX, int TY>
int ens_launch_tile(icm_ensemble *e, int mode, int grid, const void *d_cases, const EnsLaunch &L)
{
    switch (mode) {
    case kModeP2GOnly: return ens_launch_one<Pol, TX, TY, kModeP2GOnly>(e, grid, d_cases, L);
    case kModeFull: return ens_launch_one<Pol, TX, TY, kModeFull>(e, grid, d_cases, L);
    default: return ens_launch_one<Pol, TX, TY, kModeFinal>(e, grid, d_cases, L);
    }
}

template <class Pol>
int ens_launch_variant(icm_ensemble *e, int mode, int grid, const void *d_cases, const EnsLaunch &L)
{
    switch (e->variant) {
    case 0: return ens_launch_tile<Pol, 16, 8>(e, mode, grid, d_cases, L);
    case 1: return ens_launch_tile<Pol, 16, 16>(e, mode, grid, d_cases, L);
    case 2: return ens_launch_tile<Pol, 32, 8>(e, mode, grid, d_cases, L);
    default: return ens_launch_tile<Pol, 32, 16>(e, mode, grid, d_cases, L);
    }
}

int ens_launch(icm_ensemble *e, int mode, int grid, int j)
{
    EnsLaunch L{e->d_seg_base, j, e->d_tile_case, e->d_tile_local, e->d_nactive};
    if (e->form == ICM_FORM_FP64) return ens_launch_variant<Pol64>(e, mode, grid, e->d_cases, L);
    if (e->form == ICM_FORM_FP32_SURROGATE) return ens_launch_variant<Pol32S>(e, mode, grid, e->d_cases, L);
    return ens_launch_variant<Pol32>(e, mode, grid, e->d_cases, L);
}

// e->stream waits for the cases' streams (to = true) or they for it
int ens_join(icm_ensemble *e, bool to_ensemble)
{
    const size_t nc = e->cases.size();
    if (to_ensemble) {
        for (size_t i = 0; i < nc; i++) {
            ICM_CUDA(cudaEventRecord(e->events[i], e->cases[i]->stream));
            ICM_CUDA(cudaStreamWaitEvent(e->stream, e->events[i], 0));
        }
    } else {
        ICM_CUDA(cudaEventRecord(e->events[nc], e->stream));
        for (size_t i = 0; i < nc; i++) ICM_CUDA(cudaStreamWaitEvent(e->cases[i]->stream, e->events[nc], 0));
    }
    return ICM_OK;
}

template <class Pol>
int ens_upload_cases(icm_ensemble *e, const std::vector<icy_SimParams> &P, icy_SimParams *const *p, int n)
{
    const size_t nc = e->cases.size();
    std::vector<EnsCase<Pol>> hc(nc);
    for (size_t i = 0; i < nc; i++) {
        icm_ctx *c = e->cases[i];
        EnsCase<Pol> &d = hc[i];
        std::memset(&d, 0, sizeof(d));
        d.P = P[i];
        if constexpr (std::is_same<Pol, Pol64>::value) {
            d.K = Pol64::Consts{0};
            d.A = c->fz.p64;
        } else {
            d.K = make_consts32(P[i]);
            d.A = c->fz.p32;
            if (c->d_harvest && c->harvest_every > 0) {
                d.K.harvest = c->d_harvest;
                d.K.harvest_n = c->d_harvest_n;
                d.K.harvest_cap = c->harvest_cap;
                d.harvest_every = c->harvest_every;
            }
            if constexpr (std::is_same<Pol, Pol32S>::value) {
                // each case its own network, tolerance and counters
                d.K.mlp = c->d_mlp;
                d.K.mlp_tol = c->mlp_tol;
                d.K.mlp_counts = c->d_mlp_counts;
            }
        }
        TileGeom g;
        int ntiles;
        geometry(P[i], e->variant, g, ntiles);
        d.R.ntx = g.ntx;
        d.R.nty = g.nty;
        d.R.tile_start = c->bin.tile_start;
        for (int b = 0; b < 3; b++) {
            d.R.dirty[b] = c->fz.dirty + (size_t)b * ntiles;
            d.R.grid[b] = c->fz.grid[b];
        }
        d.R.bins = c->d_bins;
        d.R.err = c->d_err;
        d.R.fp64_redo = c->d_redo;
        d.R.cell_start = c->bin.cell_start;
        d.R.lane_cell = c->bin.lane_cell;
        d.R.group_base = c->bin.group_base;
        d.R.strays = c->d_strays;
        d.R.ind_y = p[i]->indenter_y;
        d.R.cost = c->fz.cost;
        d.R.tmap = c->tmap_ok ? c->d_tmap : nullptr;
        d.hist = c->d_hist;
        d.ind_x = e->d_ind_x + (size_t)i * n;
        d.active = e->d_active + e->active_off[i];
        d.step0 = p[i]->SimulationStep;
        d.every = p[i]->UpdateEveryNthStep;
        d.ntiles = ntiles;
    }
    const size_t bytes = sizeof(EnsCase<Pol>) * nc;
    if (bytes > e->cases_bytes) {
        if (e->d_cases) cudaFree(e->d_cases);
        ens_drop_graph(e);
        e->d_cases = nullptr;
        if (cudaMalloc(&e->d_cases, bytes) != cudaSuccess) return icm::fail(ICM_ERR_NOMEM, "ensemble: descriptors");
        e->cases_bytes = bytes;
    }
    ICM_CUDA(cudaMemcpyAsync(e->d_cases, hc.data(), bytes, cudaMemcpyHostToDevice, e->stream));
    return ICM_OK;
}

// Active tiles: those holding particles, their eight neighbours (the nodes
// their particles scatter to until the next re-binning) and any tile with a
// dirty flag (its nodes still need zeroing or an update). The launch list
// puts the tiles of all cases in descending order of the cost their last
// full launch measured, so the heaviest (contact, crushed zones) start
// first.
int ens_active_tiles(icm_ensemble *e, const std::vector<icy_SimParams> &P)
{
    struct Item {
        unsigned cost;
        int c, t;
    };
    const size_t nc = e->cases.size();
    // stage every case's tile starts (ntiles + 1 ints), costs (ntiles) and
    // dirty flags (3 ntiles bytes, padded to 4) with one synchronisation
    std::vector<size_t> off(nc + 1, 0);
    std::vector<int> nt(nc);
    std::vector<TileGeom> geo(nc);
    for (size_t i = 0; i < nc; i++) {
        geometry(P[i], e->variant, geo[i], nt[i]);
        off[i + 1] = off[i] + 4 * ((size_t)nt[i] + 1) + 8 * (size_t)nt[i] + ((3 * (size_t)nt[i] + 3) & ~(size_t)3);
    }
    if (off[nc] > e->stage_cap) {
        if (e->h_stage) cudaFreeHost(e->h_stage);
        e->h_stage = nullptr;
        e->stage_cap = 0;
        if (cudaMallocHost((void **)&e->h_stage, off[nc]) != cudaSuccess) {
            e->h_stage = nullptr;
            return icm::fail(ICM_ERR_NOMEM, "ensemble: pinned staging");
        }
        e->stage_cap = off[nc];
    }
    for (size_t i = 0; i < nc; i++) {
        icm_ctx *c = e->cases[i];
        unsigned char *b = e->h_stage + off[i];
        const size_t n = (size_t)nt[i];
        ICM_CUDA(cudaMemcpyAsync(b, c->bin.tile_start, 4 * (n + 1), cudaMemcpyDeviceToHost, e->stream));
        ICM_CUDA(cudaMemcpyAsync(b + 4 * (n + 1), c->fz.cost, 8 * n, cudaMemcpyDeviceToHost, e->stream));
        ICM_CUDA(cudaMemcpyAsync(b + 12 * n + 4, c->fz.dirty, 3 * n, cudaMemcpyDeviceToHost, e->stream));
    }
    ICM_CUDA(cudaStreamSynchronize(e->stream));
    std::vector<Item> items;
    std::vector<uint8_t> mask;
    unsigned long long busy_sum = 0;
    long long nbusy = 0;
    e->active_off.assign(nc, 0);
    for (size_t i = 0; i < nc; i++) {
        const int ntiles = nt[i];
        const TileGeom &g = geo[i];
        const unsigned char *b = e->h_stage + off[i];
        const int *ts = reinterpret_cast<const int *>(b);
        const unsigned *cost = reinterpret_cast<const unsigned *>(b + 4 * ((size_t)ntiles + 1));  // two halves
        const uint8_t *dirty = b + 12 * (size_t)ntiles + 4;
        e->active_off[i] = mask.size();
        mask.resize(mask.size() + (size_t)ntiles, 0);
        uint8_t *busy = mask.data() + e->active_off[i];
        for (int t = 0; t < ntiles; t++) {
            if (dirty[t] | dirty[(size_t)ntiles + t] | dirty[2 * (size_t)ntiles + t]) busy[t] = 1;
            if (ts[t + 1] == ts[t]) continue;
            const int tx = t % g.ntx, ty = t / g.ntx;
            for (int dy = -1; dy <= 1; dy++)
                for (int dx = -1; dx <= 1; dx++) {
                    const int x = tx + dx, y = ty + dy;
                    if (x >= 0 && y >= 0 && x < g.ntx && y < g.nty) busy[(size_t)y * g.ntx + x] = 1;
                }
        }
        for (int t = 0; t < ntiles; t++)
            if (busy[t]) {
                // a tile without particles (its cost may be one measured
                // before a re-binning emptied it) sorts last and is never split
                const bool has_pts = ts[t + 1] > ts[t];
                const unsigned long long cc = has_pts ? (unsigned long long)cost[t] + cost[(size_t)ntiles + t] : 0ull;
                items.push_back({cc > 0xffffffffull ? 0xffffffffu : (unsigned)cc, (int)i, t});
                if (has_pts) {
                    busy_sum += cc;
                    nbusy++;
                }
            }
    }
    // the heaviest tiles (cost above split_ratio times the mean over tiles
    // with particles, at most split_max) run as two CTAs, as in single runs
    std::stable_sort(items.begin(), items.end(), [](const Item &a, const Item &b) { return a.cost > b.cost; });
    if (nbusy > 0 && e->split_max > 0) {
        const double thr = e->split_ratio * (double)busy_sum / (double)nbusy;
        const size_t lim = std::min(items.size(), (size_t)e->split_max);
        size_t S = 0;
        while (S < lim && (double)items[S].cost > thr) S++;
        std::vector<Item> second(S);
        for (size_t k = 0; k < S; k++) {
            items[k].cost /= 2;
            items[k].t |= kSplitBit;
            second[k] = {items[k].cost, items[k].c, items[k].t | kHalfBit};
        }
        items.insert(items.end(), second.begin(), second.end());
        std::stable_sort(items.begin(), items.end(), [](const Item &a, const Item &b) { return a.cost > b.cost; });
    }
    std::vector<int> tc(items.size()), tl(items.size());
    for (size_t k = 0; k < items.size(); k++) {
        tc[k] = items[k].c;
        tl[k] = items[k].t;
    }
    const size_t m = items.size();
    int rc;
    if (m > e->tiles_cap) {
        dfree(e->d_tile_case);
        dfree(e->d_tile_local);
        ens_drop_graph(e);
        if ((rc = dalloc(&e->d_tile_case, m)) || (rc = dalloc(&e->d_tile_local, m))) return rc;
        e->tiles_cap = m;
    }
    if (mask.size() > e->active_cap) {
        dfree(e->d_active);
        if ((rc = dalloc(&e->d_active, mask.size()))) return rc;
        e->active_cap = mask.size();
    }
    e->nactive = (int)m;
    if (m) {
        ICM_CUDA(cudaMemcpyAsync(e->d_tile_case, tc.data(), sizeof(int) * m, cudaMemcpyHostToDevice, e->stream));
        ICM_CUDA(cudaMemcpyAsync(e->d_tile_local, tl.data(), sizeof(int) * m, cudaMemcpyHostToDevice, e->stream));
    }
    if (!mask.empty()) ICM_CUDA(cudaMemcpyAsync(e->d_active, mask.data(), mask.size(), cudaMemcpyHostToDevice, e->stream));
    ICM_CUDA(cudaMemcpyAsync(e->d_nactive, &e->nactive, sizeof(int), cudaMemcpyHostToDevice, e->stream));
    ICM_CUDA(cudaStreamSynchronize(e->stream));  // the host vectors go out of scope
    return ICM_OK;
}

int ens_upload(icm_ensemble *e, const std::vector<icy_SimParams> &P, icy_SimParams *const *p, int n)
{
    const int rc = ens_active_tiles(e, P);
    if (rc) return rc;
    if (e->form == ICM_FORM_FP64) return ens_upload_cases<Pol64>(e, P, p, n);
    if (e->form == ICM_FORM_FP32_SURROGATE) return ens_upload_cases<Pol32S>(e, P, p, n);
    return ens_upload_cases<Pol32>(e, P, p, n);
}

int ens_check(icm_ensemble *e)
{
    const int nc = (int)e->cases.size();
    if (e->form == ICM_FORM_FP64)
        k_ens_check<Pol64><<<nc, 128, 0, e->stream>>>(static_cast<const EnsCase<Pol64> *>(e->d_cases));
    else if (e->form == ICM_FORM_FP32_SURROGATE)
        k_ens_check<Pol32S><<<nc, 128, 0, e->stream>>>(static_cast<const EnsCase<Pol32S> *>(e->d_cases));
    else
        k_ens_check<Pol32><<<nc, 128, 0, e->stream>>>(static_cast<const EnsCase<Pol32> *>(e->d_cases));
    ICM_LAUNCHED("k_ens_check");
    return ICM_OK;
}

// A replayable segment: len full-substep launches reading their substep
// index from d_seg_base, over the current launch list (CTAs past *nactive
// return, so a graph captured for a longer list stays valid).
int ens_segment_graph(icm_ensemble *e, int len, cudaGraphExec_t &out)
{
    for (auto &g : e->graphs_by_len)
        if (g.len == len && g.grid >= e->nactive) {
            out = g.exec;
            return ICM_OK;
        }
    for (size_t i = 0; i < e->graphs_by_len.size(); i++)
        if (e->graphs_by_len[i].len == len || (int)e->graphs_by_len.size() >= kEnsGraphs) {
            cudaGraphExecDestroy(e->graphs_by_len[i].exec);
            e->graphs_by_len.erase(e->graphs_by_len.begin() + i);
            break;
        }
    // set the kernel's shared-memory attribute outside the capture (grid 0 launches nothing)
    int rc0 = ens_launch(e, kModeFull, 0, 0);
    if (rc0) return rc0;
    cudaGraph_t g = nullptr;
    ICM_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    int rc = ICM_OK;
    for (int j = 0; j < len && !rc; j++) rc = ens_launch(e, kModeFull, e->nactive, j);
    const cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
    if (rc) {
        if (g) cudaGraphDestroy(g);
        return rc;
    }
    if (ce != cudaSuccess) return icm::fail(ICM_ERR_CUDA, std::string("ensemble capture: ") + cudaGetErrorString(ce));
    cudaGraphExec_t ex = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) return icm::fail(ICM_ERR_CUDA, std::string("ensemble graph: ") + cudaGetErrorString(ie));
    e->graphs_by_len.push_back({ex, len, e->nactive});
    out = ex;
    return ICM_OK;
}

}  // namespace

extern "C" int icm_ensemble_destroy(icm_ensemble *e);

extern "C" int icm_ensemble_create(icm_ensemble **out, int device, int form, int tile_variant, int threads)
{
    if (!out) return icm::fail(ICM_ERR_ARG, "icm_ensemble_create: null out");
    *out = nullptr;
    if (form != ICM_FORM_FP32 && form != ICM_FORM_FP64 && form != ICM_FORM_FP32_SURROGATE)
        return icm::fail(ICM_ERR_ARG, "icm_ensemble_create: a fused form (FP32, FP64 or FP32 surrogate)");
    if (form == ICM_FORM_FP32_SURROGATE && threads > 32 * Pol32S::kWarps)
        return icm::fail(ICM_ERR_ARG, "icm_ensemble_create: surrogate form: at most 128 threads per block");
    if (tile_variant < 0 || tile_variant > 3 || threads < 32 || threads > 256 || threads % 32)
        return icm::fail(ICM_ERR_ARG, "icm_ensemble_create: tile variant 0..3, threads 32..256 in warps");
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        return icm::fail(ICM_ERR_NODEVICE, "No avaialble CUDA devices");
    if (device < 0 || device >= count) return icm::fail(ICM_ERR_ARG, "icm_ensemble_create: device index out of range");
    const TileVariant tv = kVariants[tile_variant];
    if (tv.TX * tv.TY > 32 * kMaxGroupsPerWarp * (threads / 32))
        return icm::fail(ICM_ERR_ARG, "tile too large for the block size (need threads >= TX*TY/4)");
    ICM_CUDA(cudaSetDevice(device));
    icm_ensemble *e = new icm_ensemble();
    e->device = device;
    e->form = form;
    e->variant = tile_variant;
    e->threads = threads;
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc((void **)&e->d_nactive, sizeof(int)) != cudaSuccess ||
        cudaMalloc((void **)&e->d_seg_base, sizeof(int)) != cudaSuccess) {
        icm_ensemble_destroy(e);
        return icm::fail(ICM_ERR_CUDA, "icm_ensemble_create: stream/allocation failed");
    }
    *out = e;
    return ICM_OK;
}

extern "C" int icm_ensemble_destroy(icm_ensemble *e)
{
    if (!e) return ICM_OK;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    ens_drop_graph(e);
    for (cudaEvent_t ev : e->events) cudaEventDestroy(ev);
    if (e->d_cases) cudaFree(e->d_cases);
    dfree(e->d_tile_case);
    dfree(e->d_tile_local);
    dfree(e->d_nactive);
    dfree(e->d_seg_base);
    dfree(e->d_ind_x);
    dfree(e->d_active);
    if (e->h_stage) cudaFreeHost(e->h_stage);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
    return ICM_OK;
}

extern "C" int icm_ensemble_add(icm_ensemble *e, icm_ctx *c)
{
    if (!e || !c) return icm::fail(ICM_ERR_ARG, "icm_ensemble_add: null argument");
    if (c->device != e->device) return icm::fail(ICM_ERR_ARG, "icm_ensemble_add: the case is on another device");
    if (!c->d_pts) return icm::fail(ICM_ERR_STATE, "icm_ensemble_add: the case has no arrays (icm_allocate_arrays)");
    for (icm_ctx *x : e->cases)
        if (x == c) return icm::fail(ICM_ERR_ARG, "icm_ensemble_add: case added twice");
    int rc = icm_set_form(c, e->form);
    if (rc) return rc;
    if ((rc = icm_set_tile(c, e->variant, e->threads))) return rc;
    cudaEvent_t ev;
    ICM_CUDA(cudaSetDevice(e->device));
    ICM_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    if (e->events.empty()) {
        cudaEvent_t ev2;
        ICM_CUDA(cudaEventCreateWithFlags(&ev2, cudaEventDisableTiming));
        e->events.push_back(ev2);  // the ensemble stream's, kept last
    }
    e->events.insert(e->events.end() - 1, ev);
    e->cases.push_back(c);
    return ICM_OK;
}

extern "C" int icm_ensemble_size(icm_ensemble *e) { return e ? (int)e->cases.size() : -1; }

extern "C" int icm_ensemble_set(icm_ensemble *e, int rebin_interval, int use_graphs)
{
    if (!e || rebin_interval < 0) return icm::fail(ICM_ERR_ARG, "icm_ensemble_set: bad argument");
    e->rebin_interval = rebin_interval;
    e->graphs = use_graphs != 0;
    return ICM_OK;
}

extern "C" int icm_ensemble_set_split(icm_ensemble *e, int max_tiles, double ratio)
{
    if (!e || max_tiles < 0 || !(ratio >= 0)) return icm::fail(ICM_ERR_ARG, "icm_ensemble_set_split: bad argument");
    e->split_max = max_tiles;
    e->split_ratio = ratio;
    return ICM_OK;
}

extern "C" void *icm_ensemble_stream(icm_ensemble *e) { return e ? (void *)e->stream : nullptr; }

extern "C" int icm_ensemble_run(icm_ensemble *e, icy_SimParams *const *p, int n)
{
    if (!e || !p) return icm::fail(ICM_ERR_ARG, "icm_ensemble_run: null argument");
    if (n < 1) return icm::fail(ICM_ERR_ARG, "icm_ensemble_run: n < 1");
    const size_t nc = e->cases.size();
    if (nc == 0) return icm::fail(ICM_ERR_STATE, "icm_ensemble_run: no cases");
    ICM_CUDA(cudaSetDevice(e->device));
    int rc;
    std::vector<icy_SimParams> P(nc);
    std::vector<double> ind_x(nc * (size_t)n);
    std::vector<double> t_end(nc);
    std::vector<char> any_pq(nc, 0);
    for (size_t i = 0; i < nc; i++) {
        icm_ctx *c = e->cases[i];
        if (!p[i]) return icm::fail(ICM_ERR_ARG, "icm_ensemble_run: null SimParams");
        if ((rc = check_params(c, p[i]))) return rc;
        if (c->form != e->form || c->tile_variant != e->variant || c->threads != e->threads)
            return icm::fail(ICM_ERR_STATE, "icm_ensemble_run: a case's form or tile was changed after icm_ensemble_add");
        if (e->form == ICM_FORM_FP32_SURROGATE && !c->d_mlp)
            return icm::fail(ICM_ERR_STATE, "icm_ensemble_run: surrogate form: a case without a network (icm_set_surrogate)");
        P[i] = kernel_params(c, p[i]);
        if (!c->internal_valid || c->fz.form != storage_form(c->form) || c->internal_variant != c->tile_variant) {
            if ((rc = ensure_ref(c)) || (rc = pack(c, P[i]))) return rc;
        }
        TileGeom g;
        int ntiles;
        geometry(P[i], e->variant, g, ntiles);
        const size_t nnodes = (size_t)P[i].GridX * P[i].GridY;
        const size_t node_bytes = (storage_form(c->form) == ICM_FORM_FP64) ? sizeof(Node64) : sizeof(float4);
        for (int b = 0; b < 3; b++) ICM_CUDA(cudaMemsetAsync(c->fz.grid[b], 0, node_bytes * nnodes, c->stream));
        ICM_CUDA(cudaMemsetAsync(c->fz.dirty, 0, 3 * (size_t)ntiles, c->stream));
        if ((rc = ensure_hist(c, n))) return rc;
        ICM_CUDA(cudaMemsetAsync(c->d_hist, 0, sizeof(double) * 2 * (size_t)n, c->stream));
        c->hist_n = n;
        if (c->fz.cost_variant != c->tile_variant || c->fz.cost_ntiles != ntiles) {
            ICM_CUDA(cudaMemsetAsync(c->fz.cost, 0, 2 * sizeof(unsigned) * (size_t)ntiles, c->stream));
            c->fz.cost_variant = c->tile_variant;
            c->fz.cost_ntiles = ntiles;
        }
        if ((rc = ensure_tmaps(c, P[i]))) return rc;
        // the indenter path of Model::Step (model.cpp:20-25) for every substep
        double t = p[i]->SimulationTime;
        for (int k = 1; k <= n; k++) {
            t += p[i]->InitialTimeStep;
            ind_x[i * (size_t)n + k - 1] = p[i]->indenter_x_initial + t * p[i]->IndVelocity;
            if ((p[i]->SimulationStep + k) % p[i]->UpdateEveryNthStep == 0) any_pq[i] = 1;
        }
        t_end[i] = t;
    }
    if ((rc = ens_join(e, true))) return rc;
    if (ind_x.size() > e->ind_x_cap) {
        dfree(e->d_ind_x);
        if ((rc = dalloc(&e->d_ind_x, ind_x.size()))) return rc;
        e->ind_x_cap = ind_x.size();
    }
    ICM_CUDA(cudaMemcpyAsync(e->d_ind_x, ind_x.data(), sizeof(double) * ind_x.size(), cudaMemcpyHostToDevice, e->stream));
    if ((rc = ens_upload(e, P, p, n))) return rc;  // synchronises the ensemble stream

    // prologue, full substeps in segments between re-binnings, final substep
    if ((rc = ens_launch(e, kModeP2GOnly, e->nactive, 0))) return rc;
    const int I = e->rebin_interval;
    int k = 1;
    while (k < n) {
        int end = n - 1;  // last full substep of this segment
        if (I > 0) end = std::min(end, ((k - 1) / I + 1) * I);
        const int len = end - k + 1;
        k_set_int<<<1, 1, 0, e->stream>>>(e->d_seg_base, k - 1);
        ICM_LAUNCHED("k_set_int");
        if (e->graphs && len > 1) {
            cudaGraphExec_t ex = nullptr;
            if ((rc = ens_segment_graph(e, len, ex))) return rc;
            ICM_CUDA(cudaGraphLaunch(ex, e->stream));
        } else {
            for (int j = 0; j < len; j++)
                if ((rc = ens_launch(e, kModeFull, e->nactive, j))) return rc;
        }
        k = end + 1;
        if (I > 0 && end % I == 0 && end < n) {
            // re-bin every case on its own stream, then refresh descriptors
            if ((rc = ens_check(e)) || (rc = ens_join(e, false))) return rc;
            for (size_t i = 0; i < nc; i++)
                if ((rc = rebin_begin(e->cases[i], P[i]))) return rc;
            for (size_t i = 0; i < nc; i++) ICM_CUDA(cudaStreamSynchronize(e->cases[i]->stream));
            for (size_t i = 0; i < nc; i++) {
                icm_ctx *c = e->cases[i];
                if ((rc = rebin_finish(c, P[i], c->internal_pq || any_pq[i]))) return rc;
            }
            if ((rc = ens_join(e, true))) return rc;
            if ((rc = ens_upload(e, P, p, n))) return rc;
        }
    }
    k_set_int<<<1, 1, 0, e->stream>>>(e->d_seg_base, n - 1);
    ICM_LAUNCHED("k_set_int");
    if ((rc = ens_launch(e, kModeFinal, e->nactive, 0))) return rc;
    if ((rc = ens_check(e)) || (rc = ens_join(e, false))) return rc;
    for (size_t i = 0; i < nc; i++) {
        icm_ctx *c = e->cases[i];
        p[i]->SimulationStep += n;
        p[i]->SimulationTime = t_end[i];
        p[i]->indenter_x = ind_x[i * (size_t)n + n - 1];
        c->internal_valid = true;
        c->ref_valid = false;
        c->internal_pq = c->internal_pq || any_pq[i];
    }
    return ICM_OK;
}

// ------------------------------------------------ learned projection

namespace icm {
int mlp_prepare_warp_net(const float *host_net, MlpWarpNet **out);
int mlp_label(const icy_SimParams &P, const float *d_harvest, int n, float *d_x, float *d_y, cudaStream_t s);
}  // namespace icm

extern "C" int icm_set_surrogate(icm_ctx *c, const float *net, float tolerance)
{
    if (!c) return icm::fail(ICM_ERR_ARG, "null context");
    if (net && !(tolerance > 0)) return icm::fail(ICM_ERR_ARG, "icm_set_surrogate: tolerance must be positive");
    ICM_CUDA(cudaSetDevice(c->device));
    ICM_CUDA(cudaStreamSynchronize(c->stream));
    dfree(c->d_mlp);
    if (!net) return ICM_OK;
    int rc = mlp_prepare_warp_net(net, &c->d_mlp);
    if (rc) return rc;
    if (!c->d_mlp_counts && (rc = dalloc(&c->d_mlp_counts, 2))) return rc;
    ICM_CUDA(cudaMemset(c->d_mlp_counts, 0, 2 * sizeof(unsigned long long)));
    c->mlp_tol = tolerance;
    return ICM_OK;
}

extern "C" int icm_surrogate_counts(icm_ctx *c, unsigned long long *accepted, unsigned long long *exact)
{
    if (!c || !accepted || !exact) return icm::fail(ICM_ERR_ARG, "icm_surrogate_counts: null argument");
    unsigned long long h[2] = {0, 0};
    if (c->d_mlp_counts) {
        ICM_CUDA(cudaStreamSynchronize(c->stream));
        ICM_CUDA(cudaMemcpy(h, c->d_mlp_counts, sizeof(h), cudaMemcpyDeviceToHost));
    }
    *accepted = h[0];
    *exact = h[1];
    return ICM_OK;
}

extern "C" int icm_set_harvest(icm_ctx *c, int capacity, int every)
{
    if (!c) return icm::fail(ICM_ERR_ARG, "null context");
    if (capacity < 0 || every < 0) return icm::fail(ICM_ERR_ARG, "icm_set_harvest: negative argument");
    ICM_CUDA(cudaSetDevice(c->device));
    ICM_CUDA(cudaStreamSynchronize(c->stream));
    dfree(c->d_harvest);
    c->harvest_cap = 0;
    c->harvest_every = 0;
    if (capacity == 0 || every == 0) return ICM_OK;
    int rc;
    if ((rc = dalloc(&c->d_harvest, 6 * (size_t)capacity))) return rc;
    if (!c->d_harvest_n && (rc = dalloc(&c->d_harvest_n, 1))) return rc;
    ICM_CUDA(cudaMemset(c->d_harvest_n, 0, sizeof(unsigned)));
    c->harvest_cap = (unsigned)capacity;
    c->harvest_every = every;
    return ICM_OK;
}

extern "C" int icm_harvest_pairs(icm_ctx *c, const icy_SimParams *p, float *x_out, float *y_out, int cap, int *n_out)
{
    if (!c || !p || !x_out || !y_out || !n_out || cap < 0)
        return icm::fail(ICM_ERR_ARG, "icm_harvest_pairs: bad argument");
    *n_out = 0;
    if (!c->d_harvest) return ICM_OK;
    ICM_CUDA(cudaSetDevice(c->device));
    ICM_CUDA(cudaStreamSynchronize(c->stream));
    unsigned got = 0;
    ICM_CUDA(cudaMemcpy(&got, c->d_harvest_n, sizeof(unsigned), cudaMemcpyDeviceToHost));
    const int n = (int)std::min<unsigned>(std::min(got, c->harvest_cap), (unsigned)cap);
    if (n > 0) {
        float *dx = nullptr, *dy = nullptr;
        int rc;
        if ((rc = dalloc(&dx, (size_t)n * 6)) || (rc = dalloc(&dy, (size_t)n * 3))) {
            dfree(dx);
            return rc;
        }
        const icy_SimParams P = kernel_params(c, p);
        rc = mlp_label(P, c->d_harvest, n, dx, dy, c->stream);
        if (!rc && cudaStreamSynchronize(c->stream) != cudaSuccess)
            rc = icm::fail(ICM_ERR_CUDA, "icm_harvest_pairs: labelling");
        if (!rc && (cudaMemcpy(x_out, dx, sizeof(float) * 6 * n, cudaMemcpyDeviceToHost) != cudaSuccess ||
                    cudaMemcpy(y_out, dy, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost) != cudaSuccess))
            rc = icm::fail(ICM_ERR_CUDA, "icm_harvest_pairs: copy");
        dfree(dx);
        dfree(dy);
        if (rc) return rc;
    }
    ICM_CUDA(cudaMemset(c->d_harvest_n, 0, sizeof(unsigned)));
    *n_out = n;
    return ICM_OK;
}

extern "C" int icm_host_alloc(void **ptr, size_t bytes)
{
    if (!ptr) return icm::fail(ICM_ERR_ARG, "null argument");
    ICM_CUDA(cudaMallocHost(ptr, bytes));
    return ICM_OK;
}

extern "C" int icm_host_free(void *ptr)
{
    if (ptr) ICM_CUDA(cudaFreeHost(ptr));
    return ICM_OK;
}
