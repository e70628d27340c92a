// k_tiles.cuh -- the fused substep: grid update + G2P + P2G in ONE launch.
//
// Data layout in HBM (internal, "tile order"):
//   * particles are binned by their stencil base node (int)(x/h - 0.5); base
//     nodes (cells) are keyed tile by tile (TX x TY nodes per tile, row-major
//     inside). Inside a tile the cells are put in lane order -- by particle
//     count, fullest first (lane_cell / cell_lane) -- and every 32
//     consecutive lanes form a group, so that a group's cells hold similar
//     counts. Each field is a structure-of-arrays in ELL slot order:
//     particle r of the cell at lane L of a group is slot
//     group_base + 32 r + L, with as many rounds as the group's fullest cell
//     (cells of the 4-per-cell lattice hold 4), so a warp reads one particle
//     of each of its 32 cells per coalesced vector load;
//   * the grid is three full-size node buffers G[0..2] of {m, px, py, -};
//     substep s reads G[s%3] (P2G result of substep s-1), scatters into
//     G[(s+1)%3] and zeroes G[(s+2)%3] (read by substep s-1), so no separate
//     reset or update launch is needed;
//   * dirty[b][t] flags tile t of buffer b as possibly non-zero.
//
// One CTA owns one node tile t and its particles:
//   1. zero t's nodes in G[(s+2)%3] if dirty;
//   2. grid update (v2_kernel_update_nodes, gpu_implementation5.cu:215-290)
//      of the (TX+4) x (TY+4) node region around t into shared memory: the
//      region is every node a particle of t can reach after drifting up to
//      one node from its tile. Halo nodes are recomputed by neighbouring CTAs
//      (the update is a pure function of the node); only the owner of a node
//      adds its reaction force, reduced in shared memory in FP64;
//   3. per particle G2P (v2_kernel_g2p, :294-379) from the shared velocities,
//      advection, Fe update, constitutive model, store;
//   4. P2G (v2_kernel_p2g, :148-213) of the updated particle for substep s+1.
//      Particles are walked cell by cell, one lane per cell, so the P2G sums
//      of a cell (all its particles share the 3x3 stencil) stay in registers
//      and reach the warp's shared region in 9 conflict-free steps; particles
//      whose stencil leaves the region fall back to global atomics;
//   5. the warps' shared regions are added to G[(s+1)%3] with one vector
//      atomic per touched node (red.global.add.v4.f32 in FP32) and the
//      touched tiles are flagged dirty.
// Velocity v and affine matrix Bp never leave registers between substeps;
// they are written only by the final launch of a run.
//
// The weighted sums of G2P and P2G are evaluated column by column (the
// quadratic B-spline weight is a product wx_i wy_j): G2P forms
// a_i = sum_j wy_j v_ij and b_i = sum_j wy_j (j - fy) v_ij, then
// v = sum_i wx_i a_i, Bp = 4/h sum_i [wx_i (i - fx) a_i, wx_i b_i]; P2G
// writes W_ij (m, c + S_h (i, j)^T) with S_h = h S and
// c = m v - S_h (fx, fy)^T, which equals W_ij (m, m v + S dpos_ij).
#pragma once
#include <cstdint>
#include <cuda.h>  // CUtensorMap (the type only)
#include <cuda_pipeline.h>
#include "mpm_math32.cuh"
#include "mlp.cuh"
#include "tc05.cuh"

namespace icm {

enum { kModeP2GOnly = 0, kModeFull = 1, kModeFinal = 2 };
constexpr int kMaxBins = 256;
// a CTA has at most 8 warps and each warp at most 4 groups of 32 cells, so
// a tile of TX*TY cells needs at least TX*TY/128 warps
constexpr int kMaxWarps = 8, kMaxGroupsPerWarp = 4;

struct alignas(16) Node64 { double m, px, py, pad; };

// Shared-memory P2G accumulator of one node (one private copy per warp):
// {m, px, py} in FP64; {px, py, m, -} in FP32, momentum first so that it
// sits in an aligned register pair for packed (f32x2) additions.
struct Acc64 { double m, px, py; };
__device__ __forceinline__ void acc_zero(float4 &a) { a = make_float4(0.f, 0.f, 0.f, 0.f); }
__device__ __forceinline__ void acc_zero(Acc64 &a) { a = Acc64{0, 0, 0}; }
__device__ __forceinline__ void acc_add(float4 &a, float m, float x, float y) { a.x += x; a.y += y; a.z += m; }
__device__ __forceinline__ void acc_add(Acc64 &a, double m, double x, double y) { a.m += m; a.px += x; a.py += y; }
__device__ __forceinline__ float acc_m(const float4 &a) { return a.z; }
__device__ __forceinline__ float acc_x(const float4 &a) { return a.x; }
__device__ __forceinline__ float acc_y(const float4 &a) { return a.y; }
__device__ __forceinline__ double acc_m(const Acc64 &a) { return a.m; }
__device__ __forceinline__ double acc_x(const Acc64 &a) { return a.px; }
__device__ __forceinline__ double acc_y(const Acc64 &a) { return a.py; }
// word offsets of m, px, py inside an accumulator
__device__ __forceinline__ constexpr int acc_off_m(const float4 *) { return 2; }
__device__ __forceinline__ constexpr int acc_off_x(const float4 *) { return 0; }
__device__ __forceinline__ constexpr int acc_off_y(const float4 *) { return 1; }
__device__ __forceinline__ constexpr int acc_off_m(const Acc64 *) { return 0; }
__device__ __forceinline__ constexpr int acc_off_x(const Acc64 *) { return 1; }
__device__ __forceinline__ constexpr int acc_off_y(const Acc64 *) { return 2; }

__device__ __forceinline__ float2 bcast2(float a) { return make_float2(a, a); }

// The 27 P2G sums of one cell (mass and momentum of its 3x3 stencil nodes),
// kept in registers by the lane that owns the cell. add() takes one
// particle: node (i, j) gets W_ij (m, c + S_h (i, j)^T) with
// W_ij = wx_i wy_j; flush() adds node (i, j)'s sums to an accumulator.
template <class real> struct CellSums {
    real m[9], x[9], y[9];
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int q = 0; q < 9; q++) { m[q] = 0; x[q] = 0; y[q] = 0; }
    }
    __device__ __forceinline__ void add(const real wx[3], const real wy[3], real mass, real c0, real c1, real S00,
                                        real S01, real S10, real S11)
    {
#pragma unroll
        for (int i = 0; i < 3; i++) {
            const real u0 = c0 + S00 * (real)i, u1 = c1 + S10 * (real)i;
            const real wm = wx[i] * mass;
#pragma unroll
            for (int j = 0; j < 3; j++) {
                const real W = wx[i] * wy[j];
                m[i * 3 + j] += wm * wy[j];
                x[i * 3 + j] += W * (u0 + S01 * (real)j);
                y[i * 3 + j] += W * (u1 + S11 * (real)j);
            }
        }
    }
    template <class Acc> __device__ __forceinline__ void flush(Acc &ac, int i, int j) const
    {
        Acc v = ac;
        acc_add(v, m[i * 3 + j], x[i * 3 + j], y[i * 3 + j]);
        ac = v;
    }
};

// FP32: the momentum sums of a node as one (x, y) pair and the masses of
// nodes (0, j) and (1, j) as one pair, updated with packed f32x2
// multiply-adds (two lanes of arithmetic per instruction).
template <> struct CellSums<float> {
    float2 xy[9];
    float2 m01[3];
    float m2[3];
    __device__ __forceinline__ void zero()
    {
#pragma unroll
        for (int q = 0; q < 9; q++) xy[q] = make_float2(0.f, 0.f);
#pragma unroll
        for (int j = 0; j < 3; j++) { m01[j] = make_float2(0.f, 0.f); m2[j] = 0.f; }
    }
    __device__ __forceinline__ void add(const float wx[3], const float wy[3], float mass, float c0, float c1, float S00,
                                        float S01, float S10, float S11)
    {
        const float2 c = make_float2(c0, c1), s0 = make_float2(S00, S10), s1 = make_float2(S01, S11);
        const float2 wx01 = make_float2(wx[0], wx[1]);
        float2 wyy[3];
#pragma unroll
        for (int j = 0; j < 3; j++) {
            wyy[j] = bcast2(wy[j]);
            const float2 mw = __fmul2_rn(bcast2(mass), wyy[j]);
            m01[j] = __ffma2_rn(mw, wx01, m01[j]);
            m2[j] = fmaf(mw.x, wx[2], m2[j]);
        }
#pragma unroll
        for (int i = 0; i < 3; i++) {
            const float2 u = i == 0 ? c : __ffma2_rn(bcast2((float)i), s0, c);
            const float2 wxx = bcast2(wx[i]);
#pragma unroll
            for (int j = 0; j < 3; j++) {
                const float2 uj = j == 0 ? u : __ffma2_rn(bcast2((float)j), s1, u);
                xy[i * 3 + j] = __ffma2_rn(__fmul2_rn(wxx, wyy[j]), uj, xy[i * 3 + j]);
            }
        }
    }
    __device__ __forceinline__ void flush(float4 &ac, int i, int j) const
    {
        float4 v = ac;
        const float2 s = __fadd2_rn(make_float2(v.x, v.y), xy[i * 3 + j]);
        const float mm = i == 2 ? m2[j] : (i == 0 ? m01[j].x : m01[j].y);
        ac = make_float4(s.x, s.y, v.z + mm, v.w);
    }
};

// The FP32 per-cell sums with compensated (Kahan) momentum accumulation:
// each momentum sum s carries the low-order part c that its additions lost,
// updated as y = p + c, t = s + y, c = y - (t - s), s = t (the differences
// as multiply-adds by -1, one rounding each); the flush adds s + c. The
// masses are sums of positive terms and are added plainly.
struct CellSumsComp {
    CellSums<float> b;
    float2 cxy[9];
    __device__ __forceinline__ void zero()
    {
        b.zero();
#pragma unroll
        for (int q = 0; q < 9; q++) cxy[q] = make_float2(0.f, 0.f);
    }
    __device__ __forceinline__ void add(const float wx[3], const float wy[3], float mass, float c0, float c1, float S00,
                                        float S01, float S10, float S11)
    {
        const float2 c = make_float2(c0, c1), s0 = make_float2(S00, S10), s1 = make_float2(S01, S11);
        const float2 wx01 = make_float2(wx[0], wx[1]), m1 = bcast2(-1.0f);
        float2 wyy[3];
#pragma unroll
        for (int j = 0; j < 3; j++) {
            wyy[j] = bcast2(wy[j]);
            const float2 mw = __fmul2_rn(bcast2(mass), wyy[j]);
            b.m01[j] = __ffma2_rn(mw, wx01, b.m01[j]);
            b.m2[j] = fmaf(mw.x, wx[2], b.m2[j]);
        }
#pragma unroll
        for (int i = 0; i < 3; i++) {
            const float2 u = i == 0 ? c : __ffma2_rn(bcast2((float)i), s0, c);
            const float2 wxx = bcast2(wx[i]);
#pragma unroll
            for (int j = 0; j < 3; j++) {
                const int q = i * 3 + j;
                const float2 uj = j == 0 ? u : __ffma2_rn(bcast2((float)j), s1, u);
                const float2 y = __fadd2_rn(__fmul2_rn(__fmul2_rn(wxx, wyy[j]), uj), cxy[q]);
                const float2 t = __fadd2_rn(b.xy[q], y);
                cxy[q] = __ffma2_rn(__ffma2_rn(b.xy[q], m1, t), m1, y);  // y - (t - s)
                b.xy[q] = t;
            }
        }
    }
    __device__ __forceinline__ void flush(float4 &ac, int i, int j) const
    {
        float4 v = ac;
        const int q = i * 3 + j;
        const float2 s = __fadd2_rn(make_float2(v.x, v.y), __fadd2_rn(b.xy[q], cxy[q]));
        const float mm = i == 2 ? b.m2[j] : (i == 0 ? b.m01[j].x : b.m01[j].y);
        ac = make_float4(s.x, s.y, v.z + mm, v.w);
    }
};

struct TileRun {
    int ntx, nty;
    const int *tile_start;   // ntiles + 1
    uint8_t *dirty[3];       // ntiles flags per buffer
    void *grid[3];
    int bufA, bufB, bufC;    // read / scatter / zero
    double ind_x, ind_y;
    double *bins;            // 2*n_indenter_subdivisions, accumulated
    double *force_slot;      // 2 doubles: this substep's summed reaction
    int *err;
    int record_pq;
    unsigned long long *fp64_redo;
    const int *cell_start;          // binning: cell key k holds cell_start[k+1] - cell_start[k] particles
    const int *lane_cell;           // the cell key at each lane (tile by tile, fullest cells first)
    const int *group_base;          // first slot of each group of 32 consecutive lanes
    unsigned long long *strays;     // particles that left their binned cell (count)
    // tile scheduling: CTA i runs tile order[i] (tile i when null); a full
    // substep launch writes tile t's clock cycles to cost[t]
    const int *order;
    unsigned *cost;
    // TMA descriptors of the three grid buffers in global memory, or null
    // (ensembles; a single run passes them as a kernel parameter)
    const CUtensorMap *tmap;
    // the tiles without particles, for the order's empty groups
    const int *empties;
    int nempty;
};

// the TMA descriptors of the three grid buffers, as a kernel parameter
struct TmapSet {
    CUtensorMap m[3];
};

// error word bits: 1 a particle left the grid (the reference's flag),
// 2 an ensemble case scattered outside its active tiles, 4 a tensor copy of
// a node region did not complete in time
constexpr int kErrTmaTimeout = 4;
// bit 8: a cell held more than 65,535 particles (the fused forms' per-cell
// count field); its particles beyond that were not advanced
constexpr int kErrCellOverflow = 8;

// launch-order entries of the fused kernel (k_tile_order): a tile, or a
// half of a split tile, or a group of kEmptyPerCta tiles without particles
// (kEmptyBit | group index into TileRun::empties)
constexpr int kTileMask = (1 << 28) - 1, kEmptyBit = 1 << 28, kSplitBit = 1 << 29, kHalfBit = 1 << 30;
constexpr int kEmptyPerCta = 8;
constexpr int kTmaPolls = 1 << 22;

// Copies the (RX x RY)-node region at node (rx0, ry0) of one grid buffer
// into shared memory with one 2D tensor copy; nodes outside the grid read as
// zero. The x coordinate is 4 * rx0 elements of 4 (FP32) or 8 (FP64) bytes,
// a multiple of 16 bytes for any rx0, negative ones included. Thread 0
// issues the copy; every thread of the CTA must later call tma_region_wait
// (the CTA may not exit with the copy in flight).
// (A descriptor in global memory must have been fenced for the tensor-map
// proxy by the issuing thread before this; one in kernel parameters needs
// nothing.)
__device__ __forceinline__ void tma_region_issue(const CUtensorMap *map, void *dst, int rx0, int ry0, uint32_t bytes,
                                                 uint64_t *bar)
{
    if (threadIdx.x == 0) {
        tc05::mbar_init(bar, 1);
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc05::smem_u32(bar)), "r"(bytes)
                     : "memory");
        asm volatile("cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
                     "[%4];" ::"r"(tc05::smem_u32(dst)),
                     "l"(map), "r"(4 * rx0), "r"(ry0), "r"(tc05::smem_u32(bar))
                     : "memory");
    }
}

// Waits for the copy; false (and kErrTmaTimeout raised) when it did not
// complete within the poll limit.
__device__ __forceinline__ bool tma_region_wait(uint64_t *bar, int *err)
{
    __syncthreads();  // the barrier was initialised before anyone polls it
    bool ok = __syncthreads_and(tc05::mbar_wait(bar, 0, kTmaPolls));
    if (!ok) {
        // give the copy a second chance to land before the buffer is reused
        __syncthreads_and(tc05::mbar_wait(bar, 0, kTmaPolls));
        if (threadIdx.x == 0) atomicOr(err, kErrTmaTimeout);
    }
    return ok;
}

struct Parts64 { double2 *pos; double4 *F; double *Jp; uint32_t *meta; double2 *vel; double4 *Bp; double2 *pq; };
// FP32 form: X = {fraction x, fraction y (32-bit fixed point, units of
// 2^-32 cells), cell (pack_cell bits), meta word (bits)}, one 16-byte vector,
// so that a particle's position and flags move in one copy; H = Fe - I;
// Jp = Jp_inv - 1. Strain form for Jp_inv and fixed point for the position
// keep the stored state as exact as the FP64 form's: a position fraction or
// Jp_inv rounded to float each substep moves the 1M-particle indentation to
// another outcome at 10,000 substeps (the crushing pattern bifurcates under
// perturbations of 1e-8), while H rounded to float does not.
struct Parts32 { float4 *X; float4 *H; float *Jp; float2 *vel; float4 *Bp; float2 *pq; };

__host__ __device__ __forceinline__ uint32_t pack_cell(int ix, int iy) { return (uint32_t)(uint16_t)(int16_t)ix | ((uint32_t)(uint16_t)(int16_t)iy << 16); }
__device__ __forceinline__ int cell_x(uint32_t c) { return (int)(int16_t)(uint16_t)(c & 0xffffu); }
__device__ __forceinline__ int cell_y(uint32_t c) { return (int)(int16_t)(uint16_t)(c >> 16); }
__device__ __forceinline__ float4 pack_x32(int ix, int iy, uint32_t ux, uint32_t uy, uint32_t meta)
{
    return make_float4(__uint_as_float(ux), __uint_as_float(uy), __uint_as_float(pack_cell(ix, iy)),
                       __uint_as_float(meta));
}

// Symmetric Kirchhoff stress as the P2G needs it.
template <class T> struct Tau { T t00, t01, t10, t11; };

// ---------------------------------------------------------------- policies

// FP64 reference form: absolute positions, Fe, Jp_inv in double; meta is
// the grain id (bits 0-15) and the crushed flag (bits 16-23).
struct Pol64 {
    static constexpr bool kSurrogate = false;
    static constexpr bool kHarvest = false;  // Consts has no harvest fields
    // registers per thread: three 128-thread CTAs per SM
    static constexpr int kMaxRegs = 168;
    // staging rounds per warp (the particle state of a round is copied into
    // shared memory kStages - 1 rounds ahead); three would cost the FP64
    // form its third CTA per SM
    static constexpr int kStages = 2;
    // Bp from raw node velocities, operation order of the reference
    static constexpr bool kRelativeGradient = false;
    using real = double;
    using V2 = double2;
    using Node = Node64;
    using Acc = Acc64;
    using Parts = Parts64;
    using Sums = CellSums<double>;
    struct Consts { int dummy; };
    struct Tables { int dummy; };
    struct St { double x, y; M2d F; double Jp; uint32_t meta; };
    struct Sten { int bx, by; double fx, fy, wx[3], wy[3]; };
    // one round of a warp (32 particles) staged in shared memory
    struct Stage { double4 F[32]; double2 pos[32]; double Jp[32]; uint32_t meta[32]; };

    static __device__ __forceinline__ void prefetch(const Parts &A, int p, Stage &S, int lane)
    {
        __pipeline_memcpy_async(&S.F[lane], &A.F[p], 16);
        __pipeline_memcpy_async(reinterpret_cast<char *>(&S.F[lane]) + 16, reinterpret_cast<const char *>(&A.F[p]) + 16, 16);
        __pipeline_memcpy_async(&S.pos[lane], &A.pos[p], 16);
        __pipeline_memcpy_async(&S.Jp[lane], &A.Jp[p], 8);
        __pipeline_memcpy_async(&S.meta[lane], &A.meta[p], 4);
    }
    static __device__ __forceinline__ St load_staged(const Stage &S, int lane)
    {
        St s;
        double2 x = S.pos[lane];
        double4 F = S.F[lane];
        s.x = x.x; s.y = x.y;
        s.F = {F.x, F.y, F.z, F.w};
        s.Jp = S.Jp[lane];
        s.meta = S.meta[lane];
        return s;
    }

    static __device__ __forceinline__ void init_tables(Tables &, const Consts &, int, int) {}
    static __device__ __forceinline__ Sten stencil(const icy_SimParams &P, const Consts &, const St &s)
    {
        Stencil64 t = stencil64(s.x, s.y, P.cellsize_inv);
        Sten r;
        r.bx = t.bx; r.by = t.by; r.fx = t.fx; r.fy = t.fy;
#pragma unroll
        for (int i = 0; i < 3; i++) { r.wx[i] = t.wx[i]; r.wy[i] = t.wy[i]; }
        return r;
    }
    static __device__ __forceinline__ St load(const Parts &A, int p)
    {
        St s;
        double2 x = A.pos[p];
        double4 F = A.F[p];
        s.x = x.x; s.y = x.y;
        s.F = {F.x, F.y, F.z, F.w};
        s.Jp = A.Jp[p];
        s.meta = A.meta[p];
        return s;
    }
    static __device__ __forceinline__ void node_velocity(const icy_SimParams &P, const Consts &, const Node &n, int gx,
                                                         int gy, double ix, double iy, double &v0, double &v1,
                                                         double &f0, double &f1, int &bin, bool contact)
    {
        bin = -1;
        if (n.m == 0) { v0 = 0; v1 = 0; return; }
        NodeOut o = update_node64(P, gx, gy, n.m, n.px, n.py, contact ? ix : 1e300, iy);
        v0 = o.v0; v1 = o.v1; f0 = o.f0; f1 = o.f1; bin = o.bin;
    }
    static __device__ __forceinline__ Tau<double> stress(const icy_SimParams &P, const Consts &, const St &s)
    {
        M2d t = kirchhoff64(s.F, P.mu, P.kappa);
        return {t.a00, t.a01, t.a10, t.a11};
    }
    // G2P tail: advect, Fe update, constitutive model; returns the stress of
    // the new Fe for the P2G that follows.
    static __device__ __forceinline__ Tau<double> advance(const icy_SimParams &P, const Consts &K, const Tables &, St &s,
                                                          double v0, double v1, const double B[4], double &p_tr,
                                                          double &q_tr, int &redo)
    {
        const double dt = P.InitialTimeStep;
        s.x += v0 * dt;
        s.y += v1 * dt;
        double M00 = 1 + dt * B[0], M01 = dt * B[1], M10 = dt * B[2], M11 = 1 + dt * B[3];
        M2d F = s.F;
        s.F = {M00 * F.a00 + M01 * F.a10, M00 * F.a01 + M01 * F.a11, M10 * F.a00 + M11 * F.a10, M10 * F.a01 + M11 * F.a11};
        uint8_t cr = (uint8_t)(s.meta >> 16);
        constitutive64_intact_first(P, s.F, s.Jp, cr, grain_res((int)(int16_t)(s.meta & 0xffffu)), p_tr, q_tr);
        s.meta = (s.meta & 0xffffu) | ((uint32_t)cr << 16);
        redo = 0;
        return stress(P, K, s);
    }
    static __device__ __forceinline__ void store(const Parts &A, int p, const St &s, double jp_old, uint32_t meta_old)
    {
        A.pos[p] = make_double2(s.x, s.y);
        A.F[p] = make_double4(s.F.a00, s.F.a01, s.F.a10, s.F.a11);
        if (s.Jp != jp_old) A.Jp[p] = s.Jp;
        if (s.meta != meta_old) A.meta[p] = s.meta;
    }
    static __device__ __forceinline__ double mass(const icy_SimParams &P, const Consts &) { return P.ParticleMass; }
    static __device__ __forceinline__ double h(const icy_SimParams &P, const Consts &) { return P.cellsize; }
    static __device__ __forceinline__ double four_h_inv(const icy_SimParams &P, const Consts &) { return 4. * P.cellsize_inv; }
    static __device__ __forceinline__ double stress_c(const icy_SimParams &P, const Consts &)
    {
        return (P.InitialTimeStep * P.ParticleVolume) * P.Dp_inv;
    }
};

// Appends a crushed particle's trial state (H, Jp_inv, meta word) to the
// harvest buffer of the surrogate's training data (out of line: only
// harvest substeps reach it).
static __device__ __noinline__ void harvest_state(const Consts32 &k, const M2f H, const float jpm1, const uint32_t meta)
{
    const unsigned slot = atomicAdd(k.harvest_n, 1u);
    if (slot >= k.harvest_cap) return;
    float *h = k.harvest + 6 * (size_t)slot;
    h[0] = H.a00;
    h[1] = H.a01;
    h[2] = H.a10;
    h[3] = H.a11;
    h[4] = 1.0f + jpm1;  // Jp_inv
    h[5] = __uint_as_float(meta);
}

// FP32 strain form: position = int16 cell + 32-bit fixed-point fraction,
// H = Fe - I, Jp = Jp_inv - 1; meta holds the grain's residues and the
// crushed flag (grain_meta32). The arithmetic is FP32.
struct Pol32 {
    static constexpr bool kSurrogate = false;
    static constexpr bool kHarvest = true;
    // registers per thread: four 128-thread CTAs per SM
    static constexpr int kMaxRegs = 128;
    // staging rounds per warp (the particle state of a round is copied into
    // shared memory kStages - 1 rounds ahead)
    static constexpr int kStages = 2;
    // Bp = 4/h sum W (v_i - v_c) dpos^T with v_c the stencil's centre node:
    // equal to the reference's sum since sum W dpos = 0, but free of the
    // cancellation of a large common velocity (whose FP32 residual would
    // repeat substep after substep for a slowly moving particle and add up
    // in Fe over thousands of substeps)
    static constexpr bool kRelativeGradient = true;
    using real = float;
    using V2 = float2;
    using Node = float4;
    using Acc = float4;
    using Parts = Parts32;
    using Sums = CellSums<float>;
    using Consts = Consts32;
    using Tables = GrainTables32;
    // position: cell (ix, iy) and fixed-point fraction (ux, uy) 2^-32; Jp:
    // Jp_inv - 1
    struct St { int ix, iy; uint32_t ux, uy; M2f H; float Jp; uint32_t meta; };
    struct Sten { int bx, by; float fx, fy, wx[3], wy[3]; };
    // one round of a warp (32 particles) staged in shared memory
    struct Stage { float4 H[32]; float4 X[32]; float Jp[32]; };

    static __device__ __forceinline__ void prefetch(const Parts &A, int p, Stage &S, int lane)
    {
        __pipeline_memcpy_async(&S.H[lane], &A.H[p], 16);
        __pipeline_memcpy_async(&S.X[lane], &A.X[p], 16);
        __pipeline_memcpy_async(&S.Jp[lane], &A.Jp[p], 4);
    }
    static __device__ __forceinline__ St unpack(const float4 X, const float4 H, float Jp)
    {
        St s;
        const uint32_t c = __float_as_uint(X.z);
        s.ix = cell_x(c); s.iy = cell_y(c);
        s.ux = __float_as_uint(X.x); s.uy = __float_as_uint(X.y);
        s.H = {H.x, H.y, H.z, H.w};
        s.Jp = Jp;
        s.meta = __float_as_uint(X.w);
        return s;
    }
    static __device__ __forceinline__ St load_staged(const Stage &S, int lane)
    {
        return unpack(S.X[lane], S.H[lane], S.Jp[lane]);
    }

    static __device__ __forceinline__ void init_tables(Tables &T, const Consts &K, int tid, int nthr)
    {
        grain_tables32_init(T, K, tid, nthr);
    }
    static __device__ __forceinline__ void base_of(int ic, float f, int &b, float &fr)
    {
        // reference: b = (int)(X - 0.5) (truncation), fr = X - b
        if (ic >= 1 || (ic == 0 && f >= 0.5f)) {
            if (f >= 0.5f) { b = ic; fr = f; }
            else { b = ic - 1; fr = f + 1.0f; }
        } else {
            float X = (float)ic + f;
            b = (int)(X - 0.5f);
            fr = X - (float)b;
        }
    }
    // the fixed-point fraction as a float in [0, 1] (rounded only for use)
    static __device__ __forceinline__ float frac(uint32_t u) { return __uint2float_rn(u) * 2.3283064365386963e-10f; }
    static __device__ __forceinline__ Sten stencil(const icy_SimParams &, const Consts &, const St &s)
    {
        Sten r;
        base_of(s.ix, frac(s.ux), r.bx, r.fx);
        base_of(s.iy, frac(s.uy), r.by, r.fy);
        float a0 = 1.5f - r.fx, a1 = r.fx - 1.0f, a2 = r.fx - 0.5f;
        r.wx[0] = 0.5f * a0 * a0; r.wx[1] = 0.75f - a1 * a1; r.wx[2] = 0.5f * a2 * a2;
        float b0 = 1.5f - r.fy, b1 = r.fy - 1.0f, b2 = r.fy - 0.5f;
        r.wy[0] = 0.5f * b0 * b0; r.wy[1] = 0.75f - b1 * b1; r.wy[2] = 0.5f * b2 * b2;
        return r;
    }
    static __device__ __forceinline__ St load(const Parts &A, int p) { return unpack(A.X[p], A.H[p], A.Jp[p]); }
    static __device__ __forceinline__ void node_velocity(const icy_SimParams &P, const Consts &k, const Node &n, int gx,
                                                         int gy, double ind_x, double ind_y, float &v0, float &v1,
                                                         double &f0, double &f1, int &bin, bool contact)
    {
        bin = -1;
        if (n.x == 0.0f) { v0 = 0.0f; v1 = 0.0f; return; }
        float inv_m = 1.0f / n.x;
        float a = n.y * inv_m, b = n.z * inv_m;
        b -= k.dt_g;
        float n2 = a * a + b * b;
        if (n2 > k.vmax * k.vmax) {
            float sc = k.vmax * rsqrtf(n2);
            a *= sc;
            b *= sc;
        }
        // contact geometry and reaction in FP64, only where the CTA's region
        // can reach the cylinder
        if (contact) {
            double n0 = gx * P.cellsize - ind_x, n1 = gy * P.cellsize - ind_y;
            if (n0 * n0 + n1 * n1 < P.IndRSq) {
                const double vco0 = P.IndVelocity;
                double va = a, vb = b;
                double vr0 = va - vco0, vr1 = vb;
                double z = n0 * n0 + n1 * n1;
                if (z > 0) { double nn = sqrt(z); n0 /= nn; n1 /= nn; }
                double vn = vr0 * n0 + vr1 * n1;
                if (vn < 0) {
                    double vt0 = vr0 - n0 * vn, vt1 = vr1 - n1 * vn;
                    double w0 = vco0 + vt0, w1 = vt1;
                    double mass = n.x;
                    f0 = (va - w0) * mass / P.InitialTimeStep;
                    f1 = (vb - w1) * mass / P.InitialTimeStep;
                    double angle = atan2(n0, n1) + ICM_PI;
                    angle *= P.n_indenter_subdivisions / (2 * ICM_PI);
                    int index = (int)angle;
                    index = max(index, 0);
                    index = min(index, P.n_indenter_subdivisions - 1);
                    bin = index;
                    a = (float)w0;
                    b = (float)w1;
                }
            }
        }
        if (gy <= 2) { a = 0.0f; b = 0.0f; }
        else if (gy >= P.GridY - 3 && b > 0.0f) b = 0.0f;
        if (gx <= 2 && a < 0.0f) a = 0.0f;
        else if (gx >= P.GridX - 3 && a > 0.0f) a = 0.0f;
        v0 = a; v1 = b;
    }
    static __device__ __forceinline__ Tau<float> stress(const icy_SimParams &, const Consts &k, const St &s)
    {
        Tau32 t = tau32(invariants32(s.H, k.mu, k.kappa));
        return {t.t00, t.t01, t.t01, t.t11};
    }
    // position and H of the particle after a substep
    static __device__ __forceinline__ void advect(const Consts &k, St &s, float v0, float v1, const float B[4])
    {
        // position: the displacement in cells, to 2^-32 cells, added to the
        // fixed-point fraction; carries move the cell
        const long long x = (long long)s.ux + __float2ll_rn(v0 * k.dt_h_inv * 4294967296.0f);
        const long long y = (long long)s.uy + __float2ll_rn(v1 * k.dt_h_inv * 4294967296.0f);
        s.ix += (int)(x >> 32);
        s.iy += (int)(y >> 32);
        s.ux = (uint32_t)x;
        s.uy = (uint32_t)y;
        // H_new = H + dt (C + C H)
        float c00 = k.dt * B[0], c01 = k.dt * B[1], c10 = k.dt * B[2], c11 = k.dt * B[3];
        M2f H = s.H;
        s.H.a00 = H.a00 + (c00 + (c00 * H.a00 + c01 * H.a10));
        s.H.a01 = H.a01 + (c01 + (c00 * H.a01 + c01 * H.a11));
        s.H.a10 = H.a10 + (c10 + (c10 * H.a00 + c11 * H.a10));
        s.H.a11 = H.a11 + (c11 + (c10 * H.a01 + c11 * H.a11));
    }
    // the FP64 redo of a particle that constitutive32 declines
    static __device__ __forceinline__ void via64(const icy_SimParams &P, St &s, float &p_tr, float &q_tr)
    {
        const Via64 o = constitutive32_via64(P, s.H, s.Jp, s.meta);
        s.H = o.H;
        s.Jp = o.jpm1;
        s.meta = o.meta;
        p_tr = o.p_tr;
        q_tr = o.q_tr;
    }
    // the trial state of a crushed particle, for the surrogate's training
    // set (only while k.harvest is set)
    static __device__ __forceinline__ void harvest(const Consts &k, const St &s)
    {
        if (meta32_crushed(s.meta) && k.harvest) harvest_state(k, s.H, s.Jp, s.meta);
    }
    static __device__ __forceinline__ Tau<float> advance(const icy_SimParams &P, const Consts &k, const Tables &T,
                                                         St &s, float v0, float v1, const float B[4], float &p_tr,
                                                         float &q_tr, int &redo)
    {
        advect(k, s, v0, v1, B);
        redo = 0;
        harvest(k, s);
        Tau32 t;
        if (constitutive32(k, T, s.H, s.Jp, s.meta, p_tr, q_tr, t) == kC32_NEEDS_FP64) {
            via64(P, s, p_tr, q_tr);
            redo = 1;
            return stress(P, k, s);
        }
        return {t.t00, t.t01, t.t01, t.t11};
    }
    static __device__ __forceinline__ void store(const Parts &A, int p, const St &s, float jp_old, uint32_t)
    {
        A.X[p] = pack_x32(s.ix, s.iy, s.ux, s.uy, s.meta);
        A.H[p] = make_float4(s.H.a00, s.H.a01, s.H.a10, s.H.a11);
        if (s.Jp != jp_old) A.Jp[p] = s.Jp;
    }
    static __device__ __forceinline__ float mass(const icy_SimParams &, const Consts &k) { return k.mass; }
    static __device__ __forceinline__ float h(const icy_SimParams &, const Consts &k) { return k.h; }
    static __device__ __forceinline__ float four_h_inv(const icy_SimParams &, const Consts &k) { return k.four_h_inv; }
    static __device__ __forceinline__ float stress_c(const icy_SimParams &, const Consts &k) { return k.stress_c; }
};

// out-of-line steps of the surrogate form (a crushed particle is rare; the
// hot loop keeps only the deferred state)
struct SurrogateOut { M2f H; float jpm1, p_tr, q_tr; int accepted, fp64; };

// The principal stretches s_i - 1 of a trial state from its FP32 invariants:
// s_i^2 - 1 = e_i = me +- rho, s_i - 1 = e_i / (sqrt(1 + e_i) + 1).
__device__ __forceinline__ void stretches32(const Inv32 &v, float rho, float &s0m1, float &s1m1)
{
    const float e0 = v.me + rho, e1 = v.me - rho;
    s0m1 = e0 / (sqrtf(1.0f + e0) + 1.0f);
    s1m1 = e1 / (sqrtf(1.0f + e1) + 1.0f);
}

// the network's input row (normalised features) of a crushed particle from
// the FP32 invariants of its trial state; false (nothing written) when
// det F <= 0.25, which the FP64 form takes
static __device__ __noinline__ bool surrogate_defer(const Consts32 &k, __nv_bfloat16 *row, const M2f H, const float jpm1)
{
    const Inv32 v = invariants32(H, k.mu, k.kappa);
    if (!(v.J > 0.25f)) return false;
    float s0m1, s1m1;
    stretches32(v, sqrtf(v.hd * v.hd + v.b01 * v.b01), s0m1, s1m1);
    const float x[kMlpIn] = {1e3f * s0m1, 1e3f * s1m1, 1e2f * jpm1, k.kappa * 1e-9f, k.tan_phi,
                             k.dp_qmax * 1e-7f};
#pragma unroll
    for (int j = 0; j < 8; j++) row[j] = __float2bfloat16(j < kMlpIn ? (x[j] - k.mlp->x_mu[j]) * k.mlp->x_isd[j] : 0.f);
    return true;
}

// applies the network's output y (normalised) when it meets the yield
// condition it stands for, else the exact projection (dp_map32, FP64 near
// its discontinuities); all in FP32 strain form from the trial state's
// invariants, recomputed here rather than carried through the round
static __device__ __noinline__ SurrogateOut surrogate_finish(const icy_SimParams &P, const Consts32 &k, const float *y,
                                                             const M2f H, const float jpm1, const uint32_t meta)
{
    const Inv32 v = invariants32(H, k.mu, k.kappa);
    const float rho = sqrtf(v.hd * v.hd + v.b01 * v.b01);
    float s0m1, s1m1;
    stretches32(v, rho, s0m1, s1m1);
    const float s0 = 1.0f + s0m1, s1 = 1.0f + s1m1;
    // p and q of the trial state (ComputePQ, gpu_implementation5.cu:36-44)
    const float p = -0.5f * v.s2, q = 2.0f * v.s1 * rho;
    const float ds0 = 1e-3f * (y[0] * k.mlp->y_sd[0] + k.mlp->y_mu[0]);
    const float ds1 = 1e-3f * (y[1] * k.mlp->y_sd[1] + k.mlp->y_mu[1]);
    const float tol = k.mlp_tol;
    SurrogateOut o{H, jpm1, p, q, 0, 0};
    bool ok = false, moved = false;
    if (!(p < -k.p_thr || jpm1 < 0.0f) && isfinite(ds0) && isfinite(ds1) && s0 + ds0 > 0.0f && s1 + ds1 > 0.0f) {
        const float qn = (p > k.dp_pmax) ? 0.0f : fminf((p + k.p_thr) * k.tan_phi, k.dp_qmax);
        if (q >= qn) {
            // q of the predicted stretches: mu/(s0' s1') (s0' - s1')(s0' + s1')
            const float s0n = s0 + ds0, s1n = s1 + ds1;
            const float gap = 2.0f * rho / (s0 + s1) + (ds0 - ds1);
            const float qp = k.mu / (s0n * s1n) * fabsf(gap * (s0n + s1n));
            const float dsum = ds0 * (2.0f * s0 + ds0) + ds1 * (2.0f * s1 + ds1);  // change of s0^2 + s1^2
            ok = fabsf(qp - qn) <= tol * k.dp_qmax && fabsf(dsum) <= tol * 1e-3f;
            moved = ok;
        } else {
            ok = fabsf(ds0) <= tol * 1e-3f && fabsf(ds1) <= tol * 1e-3f;
        }
    }
    if (ok) {
        if (moved) scale_principal32(o.H, v, rho, ds0 / s0, ds1 / s1);
        o.accepted = 1;
        return o;
    }
    if (!(v.J > 0.25f) || dp_map32(k, o.H, o.jpm1, v, p, q, rho) != kC32_OK) {
        const Via64 r = constitutive32_via64(P, H, jpm1, meta);
        o.H = r.H;
        o.jpm1 = r.jpm1;
        o.p_tr = r.p_tr;
        o.q_tr = r.q_tr;
        o.fp64 = 1;
    }
    return o;
}

// FP32 strain form with the learned Drucker-Prager projection (mlp.cuh).
// A crushed particle is decomposed in FP64 as in the FP32 form; instead of
// the exact projection (dp_project64) the network predicts the new
// singular values, once per round for the whole warp (advance defers the
// particle, network runs the warp, finish applies the result). The
// prediction is accepted when it satisfies the yield condition it stands
// for within mlp_tol: on the surface q = q_n+1 with the trial mean of
// sigma^2 kept (pressure kept), or unchanged when the trial state lies
// inside; otherwise, and for the hydrostatic branch (p < -p_thr or
// Jp_inv < 1, a closed form with nothing to learn), the exact map runs.
struct Pol32S : Pol32 {
    static constexpr bool kSurrogate = true;
    // two staging rounds: a third would not leave room for four CTAs per SM
    // next to the network's rows
    static constexpr int kStages = 2;
    // at most kWarps warps per CTA (128 threads) in this form
    static constexpr int kWarps = 4;
    // A particle held back for the network: slot, state after advection,
    // velocity and gradient for its P2G (its Jp_inv and meta word are still
    // the stored ones and are read back from the particle arrays). Kept in
    // shared memory, not registers, so the round's register use is the FP32
    // form's; with the network's rows the extra is 9 KB per CTA, which
    // keeps four 128-thread CTAs per SM.
    struct Held { int p; uint32_t cell, ux, uy; float H[4], v0, v1, B[4]; };
    struct Tables : GrainTables32 {
        alignas(16) unsigned char rows[kWarps][32 * 16];  // network input/output rows, one per lane
        Held held[kWarps][32];
    };
    static __device__ __forceinline__ void defer_save(Tables &T, int p, const St &s, float v0, float v1,
                                                      const float B[4], float, uint32_t)
    {
        T.held[threadIdx.x >> 5][threadIdx.x & 31] = {p, pack_cell(s.ix, s.iy), s.ux, s.uy,
                                                      {s.H.a00, s.H.a01, s.H.a10, s.H.a11}, v0, v1,
                                                      {B[0], B[1], B[2], B[3]}};
    }
    static __device__ __forceinline__ void defer_load(const Tables &T, const Parts &A, int &p, St &s, float &v0,
                                                      float &v1, float B[4], float &jp_old, uint32_t &meta_old)
    {
        const Held &h = T.held[threadIdx.x >> 5][threadIdx.x & 31];
        p = h.p;
        s.ix = cell_x(h.cell);
        s.iy = cell_y(h.cell);
        s.ux = h.ux;
        s.uy = h.uy;
        s.H = {h.H[0], h.H[1], h.H[2], h.H[3]};
        s.Jp = A.Jp[p];
        s.meta = __float_as_uint(A.X[p].w);
        v0 = h.v0;
        v1 = h.v1;
        for (int j = 0; j < 4; j++) B[j] = h.B[j];
        jp_old = s.Jp;
        meta_old = s.meta;
    }
    static __device__ __forceinline__ Tau<float> advance(const icy_SimParams &P, const Consts &k, Tables &T, St &s,
                                                         float v0, float v1, const float B[4], float &p_tr,
                                                         float &q_tr, int &redo)
    {
        advect(k, s, v0, v1, B);
        redo = 0;
        harvest(k, s);
        // a crushed particle's projection is the network's (from the FP32
        // invariants; det F <= 0.25 goes to the FP64 form)
        if (k.mlp && meta32_crushed(s.meta) &&
            surrogate_defer(k, reinterpret_cast<__nv_bfloat16 *>(T.rows[threadIdx.x >> 5] + (threadIdx.x & 31) * 16),
                            s.H, s.Jp)) {
            redo = 2;
            return {0.f, 0.f, 0.f, 0.f};
        }
        Tau32 t;
        if (constitutive32(k, T, s.H, s.Jp, s.meta, p_tr, q_tr, t) == kC32_OK) return {t.t00, t.t01, t.t01, t.t11};
        via64(P, s, p_tr, q_tr);
        redo = 1;
        return stress(P, k, s);
    }
    // warp-collective: lanes without a deferred particle feed zeros
    static __device__ __forceinline__ void network(const Consts &k, Tables &T, bool mine)
    {
        const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
        if (!mine) *reinterpret_cast<uint4 *>(T.rows[warp] + lane * 16) = make_uint4(0u, 0u, 0u, 0u);
        warp_mlp(k.mlp, T.rows[warp]);
    }
    static __device__ __forceinline__ Tau<float> finish(const icy_SimParams &P, const Consts &k, const Tables &T,
                                                        St &s, float &p_tr, float &q_tr, unsigned &accepted,
                                                        unsigned &exact, unsigned &fp64)
    {
        const SurrogateOut o =
            surrogate_finish(P, k, reinterpret_cast<const float *>(T.rows[threadIdx.x >> 5] + (threadIdx.x & 31) * 16),
                             s.H, s.Jp, s.meta);
        s.H = o.H;
        s.Jp = o.jpm1;
        p_tr = o.p_tr;
        q_tr = o.q_tr;
        accepted += o.accepted;
        exact += 1 - o.accepted;
        fp64 += o.fp64;
        return stress(P, k, s);
    }
};

// FP32 strain form with compensated per-cell momentum sums (CellSumsComp):
// the same arithmetic as Pol32 otherwise. The 18 compensation terms need
// registers beyond the FP32 form's 128, so this form runs three 128-thread
// CTAs per SM.
struct Pol32C : Pol32 {
    using Sums = CellSumsComp;
    static constexpr int kMaxRegs = 168;
};

// ------------------------------------------------------- grid node access

__device__ __forceinline__ void node_zero(Node64 *g, size_t i) { g[i] = Node64{0, 0, 0, 0}; }
__device__ __forceinline__ void node_zero(float4 *g, size_t i) { g[i] = make_float4(0.f, 0.f, 0.f, 0.f); }

__device__ __forceinline__ void node_add_global(Node64 *g, size_t i, double m, double px, double py)
{
    atomicAdd(&g[i].m, m);
    atomicAdd(&g[i].px, px);
    atomicAdd(&g[i].py, py);
}
__device__ __forceinline__ void node_add_global(float4 *g, size_t i, float m, float px, float py)
{
    atomicAdd(&g[i], make_float4(m, px, py, 0.0f));  // red.global.add.v4.f32 (sm_90+)
}

// ------------------------------------------------------------ the kernel

// Rare paths kept out of line so the hot loop stays small in the
// instruction cache: the velocity of a node outside the CTA's shared region
// (recomputed from the scatter buffer) and a scatter into global memory.
template <class T> struct Pair { T a, b; };

template <class Pol>
__device__ __noinline__ Pair<typename Pol::real> far_node_velocity(const icy_SimParams &P, const typename Pol::Consts &K,
                                                                   const typename Pol::Node *g, int gx, int gy,
                                                                   double ind_x, double ind_y)
{
    Pair<typename Pol::real> v{0, 0};
    if (gx < 0 || gy < 0 || gx >= P.GridX || gy >= P.GridY) return v;
    double f0, f1;
    int bin;
    Pol::node_velocity(P, K, g[(size_t)gy * P.GridX + gx], gx, gy, ind_x, ind_y, v.a, v.b, f0, f1, bin, true);
    return v;
}

template <class Pol, int TX, int TY>
__device__ __noinline__ int far_scatter(const int GX, const int GY, typename Pol::Node *g, uint8_t *dirty, int ntx,
                                        int gx, int by, typename Pol::real m0, typename Pol::real m1,
                                        typename Pol::real m2, typename Pol::real x0, typename Pol::real x1,
                                        typename Pol::real x2, typename Pol::real y0, typename Pol::real y1,
                                        typename Pol::real y2)
{
    const typename Pol::real cm[3] = {m0, m1, m2}, cx[3] = {x0, x1, x2}, cy[3] = {y0, y1, y2};
    int bad = 0;
    for (int j = 0; j < 3; j++) {
        int gy = by + j;
        if (gx < 0 || gy < 0 || gx >= GX || gy >= GY) { bad = 1; continue; }
        node_add_global(g, (size_t)gy * GX + gx, cm[j], cx[j], cy[j]);
        dirty[(gy / TY) * ntx + gx / TX] = 1;
    }
    return bad;
}

// G2P of a particle whose stencil leaves the CTA's node region: velocities
// recomputed from the scatter buffer node by node. Returns v and
// Bp = 4/h sum W (v_i - v_c) dpos^T (v_c = 0 unless Pol::kRelativeGradient),
// the arithmetic of the in-region path.
template <class T> struct G2POut { T v0, v1, B0, B1, B2, B3; };

template <class Pol>
__device__ __noinline__ G2POut<typename Pol::real> far_gather(const icy_SimParams &P, const typename Pol::Consts &K,
                                                              const typename Pol::Node *g, int bx, int by,
                                                              typename Pol::real fx, typename Pol::real fy,
                                                              typename Pol::real wx0, typename Pol::real wx1,
                                                              typename Pol::real wx2, typename Pol::real wy0,
                                                              typename Pol::real wy1, typename Pol::real wy2,
                                                              double ind_x, double ind_y)
{
    using real = typename Pol::real;
    const real wx[3] = {wx0, wx1, wx2}, wy[3] = {wy0, wy1, wy2};
    real vc0 = 0, vc1 = 0;
    if (Pol::kRelativeGradient) {
        Pair<real> c = far_node_velocity<Pol>(P, K, g, bx + 1, by + 1, ind_x, ind_y);
        vc0 = c.a;
        vc1 = c.b;
    }
    G2POut<real> o{0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 3; i++) {
        real a0 = 0, a1 = 0, b0 = 0, b1 = 0;
        for (int j = 0; j < 3; j++) {
            Pair<real> n = far_node_velocity<Pol>(P, K, g, bx + i, by + j, ind_x, ind_y);
            const real n0 = n.a - vc0, n1 = n.b - vc1;
            const real wyd = wy[j] * ((real)j - fy);
            a0 += wy[j] * n0;
            a1 += wy[j] * n1;
            b0 += wyd * n0;
            b1 += wyd * n1;
        }
        const real wxd = wx[i] * ((real)i - fx);
        o.v0 += wx[i] * a0;
        o.v1 += wx[i] * a1;
        o.B0 += wxd * a0;
        o.B2 += wxd * a1;
        o.B1 += wx[i] * b0;
        o.B3 += wx[i] * b1;
    }
    const real fhi = Pol::four_h_inv(P, K);
    o.B0 *= fhi;
    o.B1 *= fhi;
    o.B2 *= fhi;
    o.B3 *= fhi;
    o.v0 += vc0;  // sum W = 1
    o.v1 += vc1;
    return o;
}

// P2G of a particle whose base node is no longer its binned cell: shared
// atomics into the warp's region when the stencil lies inside it, global
// atomics beyond it. Node (i, j) gets W_ij (m, c + S_h (i, j)^T). Returns 1
// when a stencil node lies outside the grid (the contribution is dropped).
template <class Pol, int TX, int TY>
__device__ __noinline__ int stray_p2g(typename Pol::Acc *wacc, int rx0, int ry0, const int GX, const int GY,
                                      typename Pol::Node *g, uint8_t *dirty, int ntx, int bx, int by,
                                      typename Pol::real wx0, typename Pol::real wx1, typename Pol::real wx2,
                                      typename Pol::real wy0, typename Pol::real wy1, typename Pol::real wy2,
                                      typename Pol::real m, typename Pol::real c0, typename Pol::real c1,
                                      typename Pol::real S00, typename Pol::real S01, typename Pol::real S10,
                                      typename Pol::real S11)
{
    using real = typename Pol::real;
    constexpr int RX = TX + 4, RY = TY + 4;
    const real wx[3] = {wx0, wx1, wx2}, wy[3] = {wy0, wy1, wy2};
    const int lx = bx - rx0, ly = by - ry0;
    const bool inside = lx >= 0 && ly >= 0 && lx + 2 < RX && ly + 2 < RY && bx >= 0 && by >= 0 && bx + 2 < GX &&
                        by + 2 < GY;
    int bad = 0;
    for (int i = 0; i < 3; i++) {
        real cm[3], cx[3], cy[3];
        const real u0 = c0 + S00 * (real)i, u1 = c1 + S10 * (real)i;
        for (int j = 0; j < 3; j++) {
            const real W = wx[i] * wy[j];
            cm[j] = W * m;
            cx[j] = W * (u0 + S01 * (real)j);
            cy[j] = W * (u1 + S11 * (real)j);
        }
        if (inside) {
            for (int j = 0; j < 3; j++) {
                typename Pol::Acc *a = &wacc[(ly + j) * RX + lx + i];
                real *ap = reinterpret_cast<real *>(a);
                atomicAdd(ap + acc_off_m(a), cm[j]);
                atomicAdd(ap + acc_off_x(a), cx[j]);
                atomicAdd(ap + acc_off_y(a), cy[j]);
            }
        } else {
            bad |= far_scatter<Pol, TX, TY>(GX, GY, g, dirty, ntx, bx + i, by, cm[0], cm[1], cm[2], cx[0], cx[1], cx[2],
                                            cy[0], cy[1], cy[2]);
        }
    }
    return bad;
}

// The j-th group a warp takes: warps take groups in a snake order (w, then
// 2 nwarps - 1 - w, ...) so that the fullest groups, which come first, are
// spread over the warps; the halves of a split tile (part 1, 2) take the
// even and the odd groups. Returns a value >= the tile's group count when
// the warp has no j-th group.
__device__ __forceinline__ int group_of(int j, int warp, int nwarps, int part)
{
    const int m = j * nwarps + ((j & 1) ? nwarps - 1 - warp : warp);
    return part == 0 ? m : 2 * m + (part - 1);
}

// Whether a node of tile t's (TX+4) x (TY+4) region lies inside the
// indenter's circle.
template <int TX, int TY>
__device__ __forceinline__ bool region_touches_indenter(const icy_SimParams &P, const TileRun &R, int t)
{
    const int rx0 = (t % R.ntx) * TX - 1, ry0 = (t / R.ntx) * TY - 1;
    const double h = P.cellsize, r = sqrt(P.IndRSq);
    const double lox = rx0 * h, hix = (rx0 + TX + 3) * h, loy = ry0 * h, hiy = (ry0 + TY + 3) * h;
    const double cx = fmin(fmax(R.ind_x, lox), hix), cy = fmin(fmax(R.ind_y, loy), hiy);
    const double dx = cx - R.ind_x, dy = cy - R.ind_y;
    return dx * dx + dy * dy <= r * r;
}

// Dynamic shared memory of one CTA (host and kernel use the same layout):
// the warps' P2G regions (none in the final launch), then Pol::kStages
// staging rounds per warp.
template <class Pol, int MODE>
__host__ __device__ constexpr size_t tile_region_bytes(int RN, int nwarps)
{
    return (MODE == kModeFinal) ? 0 : (size_t)nwarps * RN * sizeof(typename Pol::Acc);
}
// The staging rounds share their space with the reduction of the indenter
// force (2 kMaxBins bins and the total, doubles), which is done with before
// the first round is staged.
constexpr size_t kBinsBytes = (2 * kMaxBins + 2) * sizeof(double);
template <class Pol, int MODE>
__host__ __device__ constexpr size_t tile_dyn_bytes(int RN, int nwarps)
{
    return tile_region_bytes<Pol, MODE>(RN, nwarps) +
           ((size_t)nwarps * Pol::kStages * sizeof(typename Pol::Stage) > kBinsBytes
                ? (size_t)nwarps * Pol::kStages * sizeof(typename Pol::Stage)
                : kBinsBytes);
}

// One substep of one tile (the body of k_tile_substep). Every return is
// uniform over the CTA.
template <class Pol, int TX, int TY, int MODE>
__device__ __forceinline__ void tile_body(const icy_SimParams &P, const typename Pol::Consts &K,
                                          const typename Pol::Parts &A, const TileRun &R, const int t,
                                          const CUtensorMap *tmaps, const bool tmaps_in_global, const int part,
                                          const bool pdl_wait)
{
    using real = typename Pol::real;
    using V2 = typename Pol::V2;
    using Node = typename Pol::Node;
    using Acc = typename Pol::Acc;
    constexpr int RX = TX + 4, RY = TY + 4, RN = RX * RY;
    __shared__ V2 s_v[RN];
    // one private accumulation region per warp (dynamic shared memory)
    extern __shared__ __align__(128) unsigned char s_dyn[];
    Acc *s_acc = reinterpret_cast<Acc *>(s_dyn);
    __shared__ uint64_t s_tma_bar;
    __shared__ int s_contact, s_mark[9];
    __shared__ typename Pol::Tables s_tab;
    // per lane of each of the warp's groups: its cell inside the tile
    // (bits 16-31) and the cell's particle count (bits 0-15)
    __shared__ uint32_t s_wcnt[kMaxWarps][kMaxGroupsPerWarp][32];
    __shared__ int s_wrounds[kMaxWarps][kMaxGroupsPerWarp], s_wgbase[kMaxWarps][kMaxGroupsPerWarp];

    const int tx = t % R.ntx, ty = t / R.ntx;
    const int x0 = tx * TX, y0 = ty * TY;
    const int rx0 = x0 - 1, ry0 = y0 - 1;
    const int GX = P.GridX, GY = P.GridY;
    const int p0 = R.tile_start[t], p1 = R.tile_start[t + 1];
    const int tid = threadIdx.x, nthr = blockDim.x;
    // force bins and total of the tile's contact nodes, in the staging space
    double *s_bins = reinterpret_cast<double *>(s_dyn + tile_region_bytes<Pol, MODE>(RN, nthr >> 5));
    double *s_tot = s_bins + 2 * kMaxBins;
    Node *gA = (Node *)R.grid[R.bufA];
    Node *gB = (Node *)R.grid[R.bufB];
    const unsigned FULL = 0xffffffffu;
    const int lane = tid & 31, warp = tid >> 5, nwarps = nthr >> 5;
    constexpr int CELLS = TX * TY;
    // part 0: the whole tile; parts 1 and 2: the even and the odd cell
    // groups of the tile (a heavy tile split over two CTAs). Both halves
    // update the node region; the first owns the tile's zeroing and its
    // reaction force.
    const int NGT_ = TX * TY / 32;
    // What depends only on the binning (unchanged since the last re-binning
    // or pack, both finished before this launch could start) is set up
    // before the wait for the previous substep: this warp's groups
    // (group_of, at most kMaxGroupsPerWarp) with their lanes' cells, cell
    // counts, rounds and slot bases, and the grain tables.
    int ng_w = 0;
    if (p1 > p0) {
        for (int g; (g = group_of(ng_w, warp, nwarps, part)) < NGT_; ng_w++) {
            const int c = R.lane_cell[t * CELLS + g * 32 + lane];
            int cnt = R.cell_start[c + 1] - R.cell_start[c];
            if (cnt > 0xffff) {  // beyond the count field: the cell's later particles are not advanced
                atomicOr(R.err, kErrCellOverflow);
                cnt = 0xffff;
            }
            s_wcnt[warp][ng_w][lane] = ((uint32_t)(c - t * CELLS) << 16) | (uint32_t)cnt;
            const int rounds = __reduce_max_sync(FULL, cnt);
            if (lane == 0) {
                s_wrounds[warp][ng_w] = rounds;
                s_wgbase[warp][ng_w] = R.group_base[(t * CELLS >> 5) + g];
            }
        }
        __syncwarp();
        if (MODE != kModeP2GOnly) Pol::init_tables(s_tab, K, tid, nthr);
    }
    // a full substep of a tile with particles stages its node region with
    // one tensor copy (below, after the wait); a descriptor in global memory
    // (written by a host copy before the launch) is fenced for the
    // tensor-map proxy here, so that the fence overlaps the wait
    bool staging = false;
    if constexpr (MODE == kModeFull) {
        staging = p1 > p0 && tmaps && tile_region_bytes<Pol, MODE>(RN, nthr >> 5) >= RN * sizeof(Node) &&
                  (tc05::smem_u32(s_dyn) & 127u) == 0;
        if (staging && tmaps_in_global && tid == 0)
            asm volatile("fence.proxy.tensormap::generic.acquire.gpu [%0], 128;" ::"l"(tmaps + R.bufA) : "memory");
    }
    // launched as a programmatic dependent: wait until the previous kernel
    // of the stream has completed and its writes are visible, then let the
    // next one launch (its CTAs take free slots, set up, and wait here)
    if (pdl_wait) {
        asm volatile("griddepcontrol.wait;" ::: "memory");
        asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    }
    // the node region's copy into the (not yet used) accumulation regions,
    // issued right after the wait so that it lands while the tile zeroes
    // its next-but-one buffer
    if constexpr (MODE == kModeFull) {
        if (staging) tma_region_issue(tmaps + R.bufA, s_dyn, rx0, ry0, (uint32_t)(RN * sizeof(Node)), &s_tma_bar);
    }

    // 1. zero this tile in the buffer the next substep will scatter into;
    //    the flag is cleared only after every thread has read it
    const bool zero_c = (MODE == kModeFull) && part != 2 && R.dirty[R.bufC][t];
    if (zero_c) {
        Node *gC = (Node *)R.grid[R.bufC];
        for (int k = tid; k < TX * TY; k += nthr) {
            int gx = x0 + k % TX, gy = y0 + k / TX;
            if (gx < GX && gy < GY) node_zero(gC, (size_t)gy * GX + gx);
        }
        __syncthreads();
        if (tid == 0) R.dirty[R.bufC][t] = 0;
    }
    const bool has_mass = (MODE != kModeP2GOnly) && R.dirty[R.bufA][t];
    const int np = p1 - p0;
    if (np == 0 && !has_mass) return;

    // can any node of the region touch the indenter?
    bool contact_possible = false;
    if (MODE != kModeP2GOnly) {
        contact_possible = region_touches_indenter<TX, TY>(P, R, t);
        if (contact_possible) {
            for (int k = tid; k < 2 * P.n_indenter_subdivisions; k += nthr) s_bins[k] = 0.0;
            if (tid == 0) { s_tot[0] = 0.0; s_tot[1] = 0.0; s_contact = 0; }
            __syncthreads();
        }
    }
    if (tid < 9) s_mark[tid] = 0;

    // 2. grid update of the region (velocities into shared memory)
    if (MODE != kModeP2GOnly) {
        if (np > 0) {
            const bool staged = staging && tma_region_wait(&s_tma_bar, R.err);
            const Node *s_nodes = reinterpret_cast<const Node *>(s_dyn);
            // four nodes per thread per pass: their loads are issued together
            constexpr int NB = 4;
            for (int k0 = tid; k0 < RN; k0 += NB * nthr) {
                Node nd[NB];
#pragma unroll
                for (int b = 0; b < NB; b++) {
                    const int k = k0 + b * nthr;
                    const int gx = rx0 + k % RX, gy = ry0 + k / RX;
                    if (staged) {
                        if (k < RN) nd[b] = s_nodes[k];
                    } else if (k < RN && gx >= 0 && gy >= 0 && gx < GX && gy < GY) {
                        nd[b] = gA[(size_t)gy * GX + gx];
                    }
                }
#pragma unroll
                for (int b = 0; b < NB; b++) {
                    const int k = k0 + b * nthr;
                    if (k >= RN) break;
                    const int gx = rx0 + k % RX, gy = ry0 + k / RX;
                    real v0 = 0, v1 = 0;
                    if (gx >= 0 && gy >= 0 && gx < GX && gy < GY) {
                        double f0 = 0, f1 = 0;
                        int bin;
                        Pol::node_velocity(P, K, nd[b], gx, gy, R.ind_x, R.ind_y, v0, v1, f0, f1, bin, contact_possible);
                        bool own = part != 2 && gx >= x0 && gx < x0 + TX && gy >= y0 && gy < y0 + TY;
                        if (bin >= 0 && own) {
                            atomicAdd(&s_bins[2 * bin], f0);
                            atomicAdd(&s_bins[2 * bin + 1], f1);
                            atomicAdd(&s_tot[0], f0);
                            atomicAdd(&s_tot[1], f1);
                            s_contact = 1;
                        }
                    }
                    s_v[k].x = v0;
                    s_v[k].y = v1;
                }
            }
        } else if (contact_possible && part != 2) {
            // no particles here: only the reaction of this tile's own nodes
            // (counted once, by the first half when the tile runs split)
            for (int k = tid; k < TX * TY; k += nthr) {
                const int gx = x0 + k % TX, gy = y0 + k / TX;
                if (gx < GX && gy < GY) {
                    Node n = gA[(size_t)gy * GX + gx];
                    real v0, v1;
                    double f0 = 0, f1 = 0;
                    int bin;
                    Pol::node_velocity(P, K, n, gx, gy, R.ind_x, R.ind_y, v0, v1, f0, f1, bin, true);
                    if (bin >= 0) {
                        atomicAdd(&s_bins[2 * bin], f0);
                        atomicAdd(&s_bins[2 * bin + 1], f1);
                        atomicAdd(&s_tot[0], f0);
                        atomicAdd(&s_tot[1], f1);
                        s_contact = 1;
                    }
                }
            }
        }
    }
    const int nwarps_blk = nthr >> 5;
    if (MODE == kModeFull && tmaps) __syncthreads();  // the staged region is read before it is zeroed
    if (MODE != kModeFinal)
        for (int k = tid; k < RN * nwarps_blk; k += nthr) acc_zero(s_acc[k]);
    __syncthreads();
    if (MODE != kModeP2GOnly && contact_possible && s_contact) {
        for (int k = tid; k < 2 * P.n_indenter_subdivisions; k += nthr)
            if (s_bins[k] != 0.0) atomicAdd(&R.bins[k], s_bins[k]);
        if (tid == 0 && R.force_slot) {
            atomicAdd(&R.force_slot[0], s_tot[0]);
            atomicAdd(&R.force_slot[1], s_tot[1]);
        }
        __syncthreads();  // the bins' space is staging space from here on
    }
    if (np == 0) return;

    // 3.-4. particles, one lane per grid cell. A lane walks the particles
    // binned to its cell and keeps the cell's 27 P2G sums (mass and momentum
    // of the 3x3 stencil) in registers; lanes of a warp hold distinct cells,
    // so the sums leave through 9 plain read-modify-write steps into the
    // warp's region, one warp barrier after each step (two cells a row apart
    // reach the same node in different steps). A particle whose base node is
    // no longer its binned cell (it moved since binning) scatters on its
    // own: shared atomics inside the region, global atomics beyond it.
    const real h = Pol::h(P, K), m = Pol::mass(P, K), fhi = Pol::four_h_inv(P, K), sc = Pol::stress_c(P, K);
    constexpr int kStages = Pol::kStages;
    int bad = 0;
    unsigned redo_count = 0, stray_count = 0, mlp_ok = 0, mlp_fb = 0;
    Acc *wacc = s_acc + warp * RN;
    typename Pol::Stage *stage =
        reinterpret_cast<typename Pol::Stage *>(s_dyn + tile_region_bytes<Pol, MODE>(RN, nwarps)) + kStages * warp;

    // work items (k, r): round r of the warp's k-th group (k = ng_w: none
    // left); the particle state of the item kStages - 1 ahead is copied into
    // its stage while this one computes
    auto next_item = [&](int k, int r, int &nk, int &nr) {
        nk = k;
        nr = r;
        if (k >= ng_w) return;
        nr = r + 1;
        if (nr >= s_wrounds[warp][k]) {
            nr = 0;
            nk = k + 1;
            while (nk < ng_w && s_wrounds[warp][nk] == 0) nk++;
        }
    };
    auto issue = [&](int k, int r, int st) {
        if (k < ng_w && r < (int)(s_wcnt[warp][k][lane] & 0xffffu))
            Pol::prefetch(A, s_wgbase[warp][k] + 32 * r + lane, stage[st], lane);
        __pipeline_commit();
    };
    int k = 0, r = 0, cur = 0;
    while (k < ng_w && s_wrounds[warp][k] == 0) k++;
    // the items 1 .. kStages - 1 ahead of the current one
    int qk[kStages - 1], qr[kStages - 1];
    issue(k, 0, 0);
#pragma unroll
    for (int a = 0; a < kStages - 1; a++) {
        next_item(a == 0 ? k : qk[a - 1], a == 0 ? r : qr[a - 1], qk[a], qr[a]);
        if (a < kStages - 2) issue(qk[a], qr[a], a + 1);
    }
    typename Pol::Sums sums;
    while (k < ng_w) {
        const int nk = qk[0], nr = qr[0];
        issue(qk[kStages - 2], qr[kStages - 2], (cur + kStages - 1) % kStages);
        __pipeline_wait_prior(kStages - 1);
        const uint32_t wc = s_wcnt[warp][k][lane];
        const int cl = (int)(wc >> 16);
        const int clx = cl % TX, cly = cl / TX;
        const int cbx = x0 + clx, cby = y0 + cly;  // the cell's base node
        const int cnt = (int)(wc & 0xffffu);
        // a cell whose stencil leaves the grid sends every particle down the
        // stray path, which raises the error word as v2_kernel_p2g does
        const bool cell_ok = cbx + 2 < GX && cby + 2 < GY;
        if (r == 0) sums.zero();
        // P2G of one (updated) particle: node (i, j) gets
        // W_ij (m, c + S_h (i, j)^T) with S = m Bp - dt Vp Dinv tau
        auto p2g = [&](const typename Pol::St &s, const real v0, const real v1, const real *B,
                       const Tau<real> &tau) {
            const typename Pol::Sten st = Pol::stencil(P, K, s);
            const real S00 = h * (m * B[0] - sc * tau.t00), S01 = h * (m * B[1] - sc * tau.t01);
            const real S10 = h * (m * B[2] - sc * tau.t10), S11 = h * (m * B[3] - sc * tau.t11);
            const real c0 = v0 * m - (S00 * st.fx + S01 * st.fy);
            const real c1 = v1 * m - (S10 * st.fx + S11 * st.fy);
            if (cell_ok && st.bx == cbx && st.by == cby) {
                sums.add(st.wx, st.wy, m, c0, c1, S00, S01, S10, S11);
            } else {
                stray_count++;
                bad |= stray_p2g<Pol, TX, TY>(wacc, rx0, ry0, GX, GY, gB, R.dirty[R.bufB], R.ntx, st.bx, st.by,
                                              st.wx[0], st.wx[1], st.wx[2], st.wy[0], st.wy[1], st.wy[2], m, c0, c1,
                                              S00, S01, S10, S11);
            }
        };
        // the lane's cell sums into the warp's region: 9 read-modify-write
        // steps, one warp barrier after each (two cells a row apart reach
        // the same node in different steps)
        auto flush_cell_sums = [&]() {
            const int ckey = (cly + 1) * RX + (clx + 1);
            __syncwarp();
#pragma unroll
            for (int i = 0; i < 3; i++)
#pragma unroll
                for (int j = 0; j < 3; j++) {
                    if (cnt > 0 && cell_ok) sums.flush(wacc[ckey + j * RX + i], i, j);
                    __syncwarp();
                }
        };
        bool deferred = false;
        if (r < cnt) {
            const int p = s_wgbase[warp][k] + 32 * r + lane;
            typename Pol::St s = Pol::load_staged(stage[cur], lane);
            real v0 = 0, v1 = 0, B[4] = {0, 0, 0, 0};
            Tau<real> tau;
            bool do_p2g = MODE != kModeFinal;
            if (MODE == kModeP2GOnly) {
                auto vv = A.vel[p];
                auto bb = A.Bp[p];
                v0 = vv.x; v1 = vv.y;
                B[0] = bb.x; B[1] = bb.y; B[2] = bb.z; B[3] = bb.w;
                tau = Pol::stress(P, K, s);
            } else {
                const auto jp_old = s.Jp;
                const uint32_t meta_old = s.meta;
                typename Pol::Sten st = Pol::stencil(P, K, s);
                const int lx = st.bx - rx0, ly = st.by - ry0;
                const bool inside = lx >= 0 && ly >= 0 && lx + 2 < RX && ly + 2 < RY && st.bx >= 0 && st.by >= 0 &&
                                    st.bx + 2 < GX && st.by + 2 < GY;
                if constexpr (sizeof(real) == 4) {
                    if (inside) {
                        // the same sums with (x, y) pairs in packed f32x2 arithmetic
                        const int q0 = ly * RX + lx;
                        const float2 vc = s_v[q0 + RX + 1];
                        const float2 nvc = make_float2(-vc.x, -vc.y);
                        float2 wyy[3], wyd[3], a[3], b[3];
#pragma unroll
                        for (int j = 0; j < 3; j++) {
                            wyy[j] = bcast2(st.wy[j]);
                            wyd[j] = bcast2(st.wy[j] * ((real)j - st.fy));
                        }
#pragma unroll
                        for (int i = 0; i < 3; i++) {
                            a[i] = make_float2(0.f, 0.f);
                            b[i] = make_float2(0.f, 0.f);
#pragma unroll
                            for (int j = 0; j < 3; j++) {
                                const float2 n = __fadd2_rn(s_v[q0 + j * RX + i], nvc);
                                a[i] = __ffma2_rn(wyy[j], n, a[i]);
                                b[i] = __ffma2_rn(wyd[j], n, b[i]);
                            }
                        }
                        float2 v = make_float2(0.f, 0.f), b02 = v, b13 = v;
#pragma unroll
                        for (int i = 0; i < 3; i++) {
                            const float2 wxx = bcast2(st.wx[i]), wxd = bcast2(st.wx[i] * ((real)i - st.fx));
                            v = __ffma2_rn(wxx, a[i], v);
                            b02 = __ffma2_rn(wxd, a[i], b02);
                            b13 = __ffma2_rn(wxx, b[i], b13);
                        }
                        const float2 f2 = bcast2(fhi);
                        b02 = __fmul2_rn(b02, f2);
                        b13 = __fmul2_rn(b13, f2);
                        v = __fadd2_rn(v, vc);  // sum W = 1
                        v0 = v.x; v1 = v.y;
                        B[0] = b02.x; B[1] = b13.x; B[2] = b02.y; B[3] = b13.y;
                    } else {
                        const G2POut<real> o = far_gather<Pol>(P, K, gA, st.bx, st.by, st.fx, st.fy, st.wx[0],
                                                               st.wx[1], st.wx[2], st.wy[0], st.wy[1], st.wy[2],
                                                               R.ind_x, R.ind_y);
                        v0 = o.v0; v1 = o.v1;
                        B[0] = o.B0; B[1] = o.B1; B[2] = o.B2; B[3] = o.B3;
                    }
                } else if (inside) {
                    real a[3][2], b[3][2];
                    real vc0 = 0, vc1 = 0;  // reference velocity of the relative form
                    const int q0 = ly * RX + lx;
                    if (Pol::kRelativeGradient) {
                        const V2 c = s_v[q0 + RX + 1];
                        vc0 = c.x;
                        vc1 = c.y;
                    }
#pragma unroll
                    for (int i = 0; i < 3; i++) {
                        a[i][0] = 0; a[i][1] = 0; b[i][0] = 0; b[i][1] = 0;
#pragma unroll
                        for (int j = 0; j < 3; j++) {
                            const V2 n = s_v[q0 + j * RX + i];
                            const real n0 = n.x - vc0, n1 = n.y - vc1;
                            const real wyd = st.wy[j] * ((real)j - st.fy);
                            a[i][0] += st.wy[j] * n0;
                            a[i][1] += st.wy[j] * n1;
                            b[i][0] += wyd * n0;
                            b[i][1] += wyd * n1;
                        }
                    }
#pragma unroll
                    for (int i = 0; i < 3; i++) {
                        const real wxd = st.wx[i] * ((real)i - st.fx);
                        v0 += st.wx[i] * a[i][0];
                        v1 += st.wx[i] * a[i][1];
                        B[0] += wxd * a[i][0];
                        B[2] += wxd * a[i][1];
                        B[1] += st.wx[i] * b[i][0];
                        B[3] += st.wx[i] * b[i][1];
                    }
                    B[0] *= fhi; B[1] *= fhi; B[2] *= fhi; B[3] *= fhi;
                    v0 += vc0;  // sum W = 1
                    v1 += vc1;
                } else {
                    const G2POut<real> o = far_gather<Pol>(P, K, gA, st.bx, st.by, st.fx, st.fy, st.wx[0], st.wx[1],
                                                           st.wx[2], st.wy[0], st.wy[1], st.wy[2], R.ind_x, R.ind_y);
                    v0 = o.v0; v1 = o.v1;
                    B[0] = o.B0; B[1] = o.B1; B[2] = o.B2; B[3] = o.B3;
                }
                real p_tr, q_tr;
                int redo;
                tau = Pol::advance(P, K, s_tab, s, v0, v1, B, p_tr, q_tr, redo);
                if constexpr (Pol::kSurrogate) {
                    if (redo == 2) {
                        deferred = true;
                        Pol::defer_save(s_tab, p, s, v0, v1, B, jp_old, meta_old);
                    }
                }
                if (!deferred) {
                    redo_count += redo;
                    Pol::store(A, p, s, jp_old, meta_old);
                    if (R.record_pq) A.pq[p] = {p_tr, q_tr};
                    if (MODE == kModeFinal) {
                        A.vel[p] = {v0, v1};
                        A.Bp[p] = {B[0], B[1], B[2], B[3]};
                    }
                }
            }
            if (do_p2g && !deferred) p2g(s, v0, v1, B, tau);
        }
        // surrogate form: particles whose projection the network makes were
        // held back above; the whole warp now evaluates the network
        if constexpr (Pol::kSurrogate) {
            if (__any_sync(FULL, deferred)) {
                // the sums are additive: hand them to the warp's region now so
                // that they are not held across the network's call
                if (MODE != kModeFinal) {
                    flush_cell_sums();
                    sums.zero();
                }
                Pol::network(K, s_tab, deferred);
                if (deferred) {
                    int dp;
                    typename Pol::St ds;
                    real dv0, dv1, dB[4], djp;
                    uint32_t dmeta;
                    Pol::defer_load(s_tab, A, dp, ds, dv0, dv1, dB, djp, dmeta);
                    real p_tr, q_tr;
                    const Tau<real> t2 = Pol::finish(P, K, s_tab, ds, p_tr, q_tr, mlp_ok, mlp_fb, redo_count);
                    Pol::store(A, dp, ds, djp, dmeta);
                    if (R.record_pq) A.pq[dp] = {p_tr, q_tr};
                    if (MODE == kModeFinal) {
                        A.vel[dp] = {dv0, dv1};
                        A.Bp[dp] = {dB[0], dB[1], dB[2], dB[3]};
                    }
                    if (MODE != kModeFinal) p2g(ds, dv0, dv1, dB, t2);
                }
            }
        }
        // last round of this group: its cells' sums go to the warp's region
        if (MODE != kModeFinal && nk != k) flush_cell_sums();
        k = nk;
        r = nr;
#pragma unroll
        for (int a = 0; a < kStages - 2; a++) {
            qk[a] = qk[a + 1];
            qr[a] = qr[a + 1];
        }
        next_item(qk[kStages - 2], qr[kStages - 2], qk[kStages - 2], qr[kStages - 2]);
        cur = cur + 1 == kStages ? 0 : cur + 1;
    }
    __pipeline_wait_prior(0);
    if (stray_count && R.strays) atomicAdd(R.strays, (unsigned long long)stray_count);
    if (bad) *R.err = 1;
    if (redo_count && R.fp64_redo) atomicAdd(R.fp64_redo, (unsigned long long)redo_count);
    if constexpr (Pol::kSurrogate) {
        if (mlp_ok) atomicAdd(&K.mlp_counts[0], (unsigned long long)mlp_ok);
        if (mlp_fb) atomicAdd(&K.mlp_counts[1], (unsigned long long)mlp_fb);
    }
    if (MODE == kModeFinal) return;
    __syncthreads();

    // 5. add the warps' shared regions to the scatter buffer
    for (int k = tid; k < RN; k += nthr) {
        Acc sum = s_acc[k];
        for (int w = 1; w < nwarps_blk; w++) {
            const Acc &o = s_acc[w * RN + k];
            acc_add(sum, acc_m(o), acc_x(o), acc_y(o));
        }
        real mm = acc_m(sum);
        if (mm == 0) continue;
        int gx = rx0 + k % RX, gy = ry0 + k / RX;
        if (gx < 0 || gy < 0 || gx >= GX || gy >= GY) continue;  // unreachable: such stencils take the fallback
        node_add_global(gB, (size_t)gy * GX + gx, mm, acc_x(sum), acc_y(sum));
        int dtx = gx / TX - tx + 1, dty = gy / TY - ty + 1;
        s_mark[dty * 3 + dtx] = 1;
    }
    __syncthreads();
    if (tid < 9 && s_mark[tid]) {
        int ntx2 = tx + tid % 3 - 1, nty2 = ty + tid / 3 - 1;
        if (ntx2 >= 0 && nty2 >= 0 && ntx2 < R.ntx && nty2 < R.nty) R.dirty[R.bufB][nty2 * R.ntx + ntx2] = 1;
    }
}

// Tiles without particles, kEmptyPerCta of them per CTA (an empty group of
// the launch order). Each one's nodes in the next-but-one buffer are zeroed
// where its dirty flag says so, and a tile that holds mass and that the
// indenter can reach adds the reaction of its own nodes (the grid update's
// contact, gpu_implementation5.cu:245-271) to the force bins with global
// FP64 atomics. The group's flags are read at once, after the wait for the
// previous substep, so that the latency of the loads is paid once per CTA.
template <class Pol, int TX, int TY, int MODE>
__device__ __forceinline__ void empty_group(const icy_SimParams &P, const typename Pol::Consts &K, const TileRun &R,
                                            const int grp)
{
    using Node = typename Pol::Node;
    using real = typename Pol::real;
    __shared__ int s_et[kEmptyPerCta];
    __shared__ uint8_t s_ez[kEmptyPerCta], s_ec[kEmptyPerCta];
    const int tid = threadIdx.x, nthr = blockDim.x;
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    if (tid < kEmptyPerCta) {
        const int i = grp * kEmptyPerCta + tid;
        int t = -1;
        uint8_t z = 0, c = 0;
        if (i < R.nempty) {
            t = R.empties[i];
            z = (MODE == kModeFull) ? R.dirty[R.bufC][t] : 0;
            c = (R.dirty[R.bufA][t] && region_touches_indenter<TX, TY>(P, R, t)) ? 1 : 0;
        }
        s_et[tid] = t;
        s_ez[tid] = z;
        s_ec[tid] = c;
    }
    __syncthreads();
    const int GX = P.GridX, GY = P.GridY;
    for (int j = 0; j < kEmptyPerCta; j++) {
        const int t = s_et[j];
        if (t < 0) continue;
        const int x0 = (t % R.ntx) * TX, y0 = (t / R.ntx) * TY;
        if (s_ez[j]) {
            Node *gC = (Node *)R.grid[R.bufC];
            for (int k = tid; k < TX * TY; k += nthr) {
                const int gx = x0 + k % TX, gy = y0 + k / TX;
                if (gx < GX && gy < GY) node_zero(gC, (size_t)gy * GX + gx);
            }
        }
        if (s_ec[j]) {
            const Node *gA = (const Node *)R.grid[R.bufA];
            for (int k = tid; k < TX * TY; k += nthr) {
                const int gx = x0 + k % TX, gy = y0 + k / TX;
                if (gx >= GX || gy >= GY) continue;
                real v0, v1;
                double f0 = 0, f1 = 0;
                int bin;
                Pol::node_velocity(P, K, gA[(size_t)gy * GX + gx], gx, gy, R.ind_x, R.ind_y, v0, v1, f0, f1, bin, true);
                if (bin >= 0) {
                    atomicAdd(&R.bins[2 * bin], f0);
                    atomicAdd(&R.bins[2 * bin + 1], f1);
                    if (R.force_slot) {
                        atomicAdd(&R.force_slot[0], f0);
                        atomicAdd(&R.force_slot[1], f1);
                    }
                }
            }
        }
    }
    __syncthreads();  // every thread's zeroing is done before the flags clear
    if (tid < kEmptyPerCta && s_et[tid] >= 0 && s_ez[tid]) R.dirty[R.bufC][s_et[tid]] = 0;
}

// One launch = one substep over all tiles, one CTA per tile. Tile costs are
// uneven (indenter contact, crushed particles redone in FP64, occupancy), so
// CTA i takes tile order[i] -- the tiles sorted by the cost measured in
// earlier launches, heaviest first, which the hardware dispatches first --
// instead of letting late heavy tiles form the tail of the launch.
template <class Pol, int TX, int TY, int MODE>
__global__ void __maxnreg__(Pol::kMaxRegs) k_tile_substep(const __grid_constant__ icy_SimParams P,
                                                      const __grid_constant__ typename Pol::Consts K,
                                                      const typename Pol::Parts A, const __grid_constant__ TileRun R,
                                                      const __grid_constant__ TmapSet T)
{
    __shared__ long long s_clock;
    const int ntiles = R.ntx * R.nty;
    // order entries: tile | split << 29 | second half << 30, or -1 (nothing)
    int code;
    if (R.order) {
        code = R.order[blockIdx.x];
    } else {
        code = (int)blockIdx.x < ntiles ? (int)blockIdx.x : -1;
    }
    if (code < 0) return;
    if (code & kEmptyBit) {
        // the prologue (P2G of the current state) has nothing to do there
        if (MODE != kModeP2GOnly) empty_group<Pol, TX, TY, MODE>(P, K, R, code & kTileMask);
        return;
    }
    const int t = code & kTileMask;
    const int part = (code & kSplitBit) ? ((code & kHalfBit) ? 2 : 1) : 0;
    if (MODE == kModeFull && threadIdx.x == 0) s_clock = clock64();
    tile_body<Pol, TX, TY, MODE>(P, K, A, R, t, R.tmap ? T.m : nullptr, false, part, true);
    if (MODE == kModeFull && R.cost) {
        __syncthreads();
        if (threadIdx.x == 0) {
            // cost[t] and cost[ntiles + t]: the tile's two halves (the second
            // is zero for a tile run whole)
            const long long dc = clock64() - s_clock;
            const unsigned c = (unsigned)(dc < 0 ? 0 : (dc > 0xffffffffll ? 0xffffffffll : dc));
            R.cost[part == 2 ? ntiles + t : t] = c;
            if (part == 0) R.cost[ntiles + t] = 0;
        }
    }
}

// ---------------------------------------------------------- ensembles
// Many cases (separate blocks, materials and indenters, each with its own
// grid and particle arrays) advance together: one launch per substep covers
// the active tiles of every case. A case's parameter block, constants,
// particle arrays and the fixed part of its TileRun are read by each of its
// CTAs into shared memory; everything that changes from substep to substep
// is derived on the device from the substep index sidx = *seg_base + j, so
// that one captured sequence of launches can be replayed for any segment.
template <class Pol> struct EnsCase {
    icy_SimParams P;
    typename Pol::Consts K;
    typename Pol::Parts A;
    TileRun R;
    double *hist;          // 2 doubles per substep of the run
    const double *ind_x;   // indenter x after each substep of the run
    const uint8_t *active; // 1 for each tile this case's launches cover
    int step0, every;      // SimulationStep when the run started, UpdateEveryNthStep
    int ntiles;
    int harvest_every;     // FP32 form: substeps between harvests of crushed states (0: none)
};

// the harvest pointer of a launch that is not a harvest substep is cleared
template <class Pol> __device__ __forceinline__ void ens_gate_harvest(EnsCase<Pol> &c, int sidx, bool on)
{
    if constexpr (Pol::kHarvest) {
        if (!(on && c.harvest_every > 0 && (c.step0 + sidx + 1) % c.harvest_every == 0)) c.K.harvest = nullptr;
    }
}

struct EnsLaunch {
    const int *seg_base;   // substep index of the first launch of the segment
    int j;                 // this launch's place in the segment
    const int *tile_case;  // active tiles: case and tile within the case
    const int *tile_local;
    const int *nactive;    // number of active tiles (CTAs past it return)
};

template <class Pol, int TX, int TY, int MODE>
__global__ void __maxnreg__(Pol::kMaxRegs) k_tile_substep_ens(const EnsCase<Pol> *__restrict__ cases,
                                                                           const __grid_constant__ EnsLaunch L)
{
    __shared__ __align__(16) EnsCase<Pol> sc;
    __shared__ long long s_clock;
    // a programmatic dependent of the previous substep (see k_tile_substep):
    // the launch list, the case descriptors and the segment's first substep
    // index are written before the segment starts, so they are read before
    // tile_body waits for the previous substep
    if ((int)blockIdx.x >= *L.nactive) return;
    // tile_local: tile | split << 29 | second half << 30 (as the single-run order)
    const int c = L.tile_case[blockIdx.x], code = L.tile_local[blockIdx.x];
    const int t = code & kTileMask;
    const int part = (code & kSplitBit) ? ((code & kHalfBit) ? 2 : 1) : 0;
    {
        const uint32_t *src = reinterpret_cast<const uint32_t *>(cases + c);
        uint32_t *dst = reinterpret_cast<uint32_t *>(&sc);
        for (int i = threadIdx.x; i < (int)(sizeof(EnsCase<Pol>) / 4); i += blockDim.x) dst[i] = src[i];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        if (MODE == kModeP2GOnly) {
            sc.R.bufA = sc.R.bufB = sc.R.bufC = 0;
            sc.R.force_slot = nullptr;
            sc.R.record_pq = 0;
            sc.R.ind_x = sc.P.indenter_x;
            ens_gate_harvest(sc, 0, false);
        } else {
            const int sidx = *L.seg_base + L.j;
            sc.R.bufA = sidx % 3;
            sc.R.bufB = (sidx + 1) % 3;
            sc.R.bufC = (sidx + 2) % 3;
            sc.R.ind_x = sc.ind_x[sidx];
            sc.R.force_slot = sc.hist + 2 * (size_t)sidx;
            sc.R.record_pq = (sc.step0 + sidx + 1) % sc.every == 0 ? 1 : 0;
            ens_gate_harvest(sc, sidx, true);
            s_clock = clock64();
        }
    }
    __syncthreads();
    tile_body<Pol, TX, TY, MODE>(sc.P, sc.K, sc.A, sc.R, t, sc.R.tmap, true, part, true);
    if (MODE == kModeFull && sc.R.cost) {
        __syncthreads();
        if (threadIdx.x == 0) {
            const long long dc = clock64() - s_clock;
            const unsigned cc = (unsigned)(dc < 0 ? 0 : (dc > 0xffffffffll ? 0xffffffffll : dc));
            sc.R.cost[part == 2 ? sc.ntiles + t : t] = cc;
            if (part == 0) sc.R.cost[sc.ntiles + t] = 0;
        }
    }
}

__global__ void k_set_int(int *dst, int value) { *dst = value; }

// After a segment: a tile outside a case's active set whose dirty flag is
// set received mass that no launch consumed (a particle drifted further
// than a tile between re-binnings). Sets bit 2 of the case's error word.
template <class Pol> __global__ void k_ens_check(const EnsCase<Pol> *__restrict__ cases)
{
    const EnsCase<Pol> &c = cases[blockIdx.x];
    bool lost = false;
    for (int t = threadIdx.x; t < c.ntiles; t += blockDim.x)
        if (!c.active[t] && (c.R.dirty[0][t] | c.R.dirty[1][t] | c.R.dirty[2][t])) lost = true;
    if (__syncthreads_or(lost) && threadIdx.x == 0) atomicOr(c.R.err, 2);
}

constexpr int kMaxOrderTiles = 8192;
constexpr int kOrderThreads = 1024;

// ------------------------------------------------ binning, pack and unpack

struct TileGeom { int TX, TY, ntx, nty; };

// base node of a reference-layout particle, clamped into the grid
__device__ __forceinline__ int sort_key(const icy_SimParams &P, const TileGeom &g, double x, double y)
{
    int bx = (int)(x * P.cellsize_inv - 0.5), by = (int)(y * P.cellsize_inv - 0.5);
    bx = min(max(bx, 0), P.GridX - 1);
    by = min(max(by, 0), P.GridY - 1);
    int tx = bx / g.TX, ty = by / g.TY;
    return ((ty * g.ntx + tx) * g.TY + (by - ty * g.TY)) * g.TX + (bx - tx * g.TX);
}

__global__ void k_bin_keys(const icy_SimParams P, const TileGeom g, int *key, int *count)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.nPts) return;
    const double *pts = P.pts_array;
    double x = pts[(size_t)ICM_IDX_POSX * P.nPtsPitch + i];
    double y = pts[(size_t)(ICM_IDX_POSX + 1) * P.nPtsPitch + i];
    int k = sort_key(P, g, x, y);
    key[i] = k;
    atomicAdd(&count[k], 1);
}

// exclusive scan, 3 phases over chunks of 4*1024 ints
constexpr int kScanThreads = 1024, kScanItems = 4, kScanChunk = kScanThreads * kScanItems;

__device__ __forceinline__ int block_exclusive_scan(int v, int *tmp, int &total)
{
    int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) tmp[w] = x;
    __syncthreads();
    if (w == 0) {
        int nw = blockDim.x >> 5;
        int s = lane < nw ? tmp[lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            int y = __shfl_up_sync(0xffffffffu, s, o);
            if (lane >= o) s += y;
        }
        if (lane < nw) tmp[lane] = s;
    }
    __syncthreads();
    int before = (w > 0 ? tmp[w - 1] : 0) + x - v;
    total = tmp[(blockDim.x >> 5) - 1];
    __syncthreads();
    return before;
}

// Launch order of the fused substep (one CTA, n <= kMaxOrderTiles): the
// tiles holding particles by descending cost, then the tiles without
// particles in groups of kEmptyPerCta (one CTA each, entries kEmptyBit |
// group, the tiles listed in empties). The cost order is a counting sort on
// the cost quantised to kOrderLevels levels of the largest cost; inside a
// level the order is the order in which threads claim places, which no
// result depends on (a substep's result does not depend on the order its
// CTAs run in). A tile's cost is cost[t] + cost[n + t] (its halves when it
// ran split). The first S tiles are split, S = the number of tiles whose
// cost exceeds ratio times the mean over tiles holding particles, at most
// max_split: their two halves lead the order (two CTAs each). The order has
// n + max_split entries, the unused ones -1; a launch needs its first
// busy + S + ceil((n - busy) / kEmptyPerCta). Dynamic shared memory: 2 n ints.
constexpr int kOrderLevels = kOrderThreads;

__global__ void __launch_bounds__(kOrderThreads) k_tile_order(int n, const unsigned *cost, const int *tile_start,
                                                              int max_split, float ratio, int *order, int *empties)
{
    extern __shared__ int s_sorted[];
    // per tile: its cost (kNoCost: no particles), then its level
    unsigned *s_c = reinterpret_cast<unsigned *>(s_sorted + n);
    constexpr unsigned kNoCost = 0xffffffffu;
    __shared__ int s_off[kOrderLevels];
    __shared__ int s_tmp[32];
    __shared__ unsigned long long s_sum;
    __shared__ unsigned s_max;
    __shared__ int s_busy, s_over;
    const unsigned FULL = 0xffffffffu;
    const int tid = threadIdx.x;
    for (int b = tid; b < kOrderLevels; b += blockDim.x) s_off[b] = 0;
    if (tid == 0) {
        s_sum = 0;
        s_max = 0;
        s_busy = 0;
        s_over = 0;
    }
    unsigned long long sum = 0;
    unsigned mx = 0;
    int busy = 0;
    for (int i = tid; i < n; i += blockDim.x) {
        unsigned c = kNoCost;
        if (tile_start[i + 1] > tile_start[i]) {
            const unsigned long long cc = (unsigned long long)cost[i] + cost[n + i];
            c = cc >= kNoCost ? kNoCost - 1 : (unsigned)cc;
            sum += c;
            busy++;
            mx = max(mx, c);
        }
        s_c[i] = c;
    }
    // one shared atomic per warp (a thousand on one address serialise, the
    // 64-bit sum as a compare-and-swap loop)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(FULL, sum, o);
    busy = __reduce_add_sync(FULL, busy);
    mx = __reduce_max_sync(FULL, mx);
    __syncthreads();  // s_off and the totals are zero
    if ((tid & 31) == 0) {
        atomicAdd(&s_sum, sum);
        atomicAdd(&s_busy, busy);
        atomicMax(&s_max, mx);
    }
    __syncthreads();
    const unsigned cmax = max(s_max, 1u);
    const int nbusy = s_busy;
    const double thr = nbusy > 0 ? (double)ratio * (double)s_sum / (double)nbusy : 1e300;
    // busy tiles take levels 1 .. kOrderLevels - 1 (the heaviest the top
    // one), tiles without particles level 0. Most tiles hold no particles
    // and share level 0: a warp adds once per distinct level (shared atomics
    // on one address serialise).
    int over = 0;
    for (int i0 = tid - (tid & 31); i0 < n; i0 += blockDim.x) {
        const int i = i0 + (tid & 31);
        int lv = -1;
        if (i < n) {
            const unsigned c = s_c[i];
            lv = 0;
            if (c != kNoCost) {
                lv = 1 + (int)((unsigned long long)c * (kOrderLevels - 2) / cmax);
                over += (double)c > thr;
            }
            s_c[i] = (unsigned)lv;
        }
        const unsigned peers = __match_any_sync(FULL, lv);
        if (lv >= 0 && (tid & 31) == __ffs(peers) - 1) atomicAdd(&s_off[lv], __popc(peers));
    }
    over = __reduce_add_sync(FULL, over);
    if ((tid & 31) == 0) atomicAdd(&s_over, over);
    __syncthreads();
    // start of each level in descending level order: thread t takes level
    // kOrderLevels - 1 - t (blockDim.x == kOrderLevels)
    {
        const int b = kOrderLevels - 1 - tid;
        int total;
        const int before = block_exclusive_scan(s_off[b], s_tmp, total);
        __syncthreads();
        s_off[b] = before;
    }
    __syncthreads();
    for (int i0 = tid - (tid & 31); i0 < n; i0 += blockDim.x) {
        const int i = i0 + (tid & 31);
        const int lv = i < n ? (int)s_c[i] : -1;
        const unsigned peers = __match_any_sync(FULL, lv);
        const int leader = __ffs(peers) - 1;
        int base = 0;
        if (lv >= 0 && (tid & 31) == leader) base = atomicAdd(&s_off[lv], __popc(peers));
        base = __shfl_sync(FULL, base, leader);
        // places in lane order within the warp's share of the level
        if (lv >= 0) s_sorted[base + __popc(peers & ((1u << (tid & 31)) - 1))] = i;
    }
    __syncthreads();
    const int S = min(min(s_over, max_split), nbusy);
    const int nempty = n - nbusy, ngroups = (nempty + kEmptyPerCta - 1) / kEmptyPerCta;
    for (int i = tid; i < nempty; i += blockDim.x) empties[i] = s_sorted[nbusy + i];
    for (int i = tid; i < n + max_split; i += blockDim.x) {
        int v = -1;
        if (i < 2 * S) {
            v = s_sorted[i >> 1] | kSplitBit | ((i & 1) ? kHalfBit : 0);
        } else if (i < nbusy + S) {
            v = s_sorted[i - S];
        } else if (i < nbusy + S + ngroups) {
            v = (i - nbusy - S) | kEmptyBit;
        }
        order[i] = v;
    }
}

__global__ void __launch_bounds__(kScanThreads) k_scan_chunks(const int *in, int n, int *chunk_sums)
{
    __shared__ int tmp[32];
    int base = blockIdx.x * kScanChunk + threadIdx.x * kScanItems;
    int s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++)
        if (base + k < n) s += in[base + k];
    int total;
    block_exclusive_scan(s, tmp, total);
    if (threadIdx.x == 0) chunk_sums[blockIdx.x] = total;
}

// One block: exclusive scan of a short array (n <= kScanThreads *
// kScanSmallItems), and out[n] = the total. Warp w takes a run of seg
// consecutive entries (seg a multiple of 32) and reads it in rows of 32
// (coalesced): once to add it up, and after the block has scanned the warps'
// sums, again to scan it row by row with warp shuffles.
constexpr int kScanSmallItems = 32;
__global__ void __launch_bounds__(kScanThreads) k_scan_small(const int *in, int n, int *out)
{
    __shared__ int tmp[32];
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int seg = (n + 32 * nw - 1) / (32 * nw) * 32;
    const int e0 = w * seg;
    int s = 0;
    for (int r = 0; r < seg; r += 32) {
        const int e = e0 + r + lane;
        if (e < n) s += in[e];
    }
    s = __reduce_add_sync(FULL, s);
    int total;
    int off = block_exclusive_scan(lane == 0 ? s : 0, tmp, total);
    off = __shfl_sync(FULL, off, 0);  // the sum of the warps before this one
#pragma unroll 4
    for (int r = 0; r < seg; r += 32) {
        const int e = e0 + r + lane;
        const int x = e < n ? in[e] : 0;
        int y = x;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int z = __shfl_up_sync(FULL, y, o);
            if (lane >= o) y += z;
        }
        if (e < n) out[e] = off + y - x;
        off += __shfl_sync(FULL, y, 31);
    }
    if (threadIdx.x == 0) out[n] = total;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_apply(const int *in, int n, const int *chunk_sums, int *out)
{
    __shared__ int tmp[32];
    int off = 0;
    for (int i = threadIdx.x; i < (int)blockIdx.x; i += blockDim.x) off += chunk_sums[i];
    {
        int total;
        block_exclusive_scan(off, tmp, total);
        off = total;
    }
    int base = blockIdx.x * kScanChunk + threadIdx.x * kScanItems;
    int v[kScanItems], s = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        v[k] = (base + k < n) ? in[base + k] : 0;
        s += v[k];
    }
    int total;
    int before = block_exclusive_scan(s, tmp, total) + off;
#pragma unroll
    for (int k = 0; k < kScanItems; k++) {
        if (base + k < n) out[base + k] = before;
        before += v[k];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) out[n] = before;
}

__global__ void k_bin_scatter(int n, const int *key, int *cursor, int *perm)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    int pos = atomicAdd(&cursor[key[i]], 1);
    perm[pos] = i;
}

// Restores particle order inside every cell (atomic scatter order is not
// deterministic): insertion sort of the few indices of each cell.
__global__ void k_bin_order(int ncells, const int *start, int *perm)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    int a = start[c], b = start[c + 1];
    for (int i = a + 1; i < b; i++) {
        int v = perm[i], j = i - 1;
        while (j >= a && perm[j] > v) { perm[j + 1] = perm[j]; j--; }
        perm[j + 1] = v;
    }
}

// Lane order of the cells of each tile (one warp per tile, cells_per_tile a
// multiple of 32 and at most kMaxTileCells): by particle count, fullest
// first, ties by cell key. lane_cell[l] is the cell key at lane l and
// cell_lane its inverse; both index the tile's own range of keys,
// t * cells_per_tile + i. A group of 32 consecutive lanes then holds cells of
// similar counts, so that few of its lanes idle through the rounds of its
// fullest cell. The same pass writes what follows from the order:
// group_slots (32 x the count of the group's first, fullest lane: its slots
// in the ELL layout), tile_start[t] (the tile's first particle; the last
// tile also writes tile_start[ntiles]) and *nbusy (tiles holding particles,
// zeroed by the caller). The warp visits the distinct counts from the
// largest down; at each it places the cells of that count in key order
// (ballots over the tile's rows of 32 keys).
constexpr int kMaxTileCells = 512, kLaneOrderWarps = 4;

__global__ void __launch_bounds__(32 * kLaneOrderWarps) k_lane_order(int ntiles, int cells_per_tile,
                                                                    const int *cell_start, int *lane_cell,
                                                                    int *cell_lane, int *group_slots,
                                                                    int *tile_start, int *nbusy)
{
    constexpr int kRows = kMaxTileCells / 32;
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int t = blockIdx.x * kLaneOrderWarps + (threadIdx.x >> 5);
    if (t >= ntiles) return;
    const int base = t * cells_per_tile, rows = cells_per_tile / 32;
    const int first = cell_start[base], last = cell_start[base + cells_per_tile];
    if (lane == 0) {
        tile_start[t] = first;
        if (t == ntiles - 1) tile_start[ntiles] = last;
        if (last > first) atomicAdd(nbusy, 1);
    }
    if (last == first) {
        // no particles: every count is 0, and the order by key is the identity
        for (int i = lane; i < cells_per_tile; i += 32) {
            lane_cell[base + i] = base + i;
            cell_lane[base + i] = base + i;
        }
        if (lane < rows) group_slots[(base >> 5) + lane] = 0;
        return;
    }
    int cnt[kRows];
    int mx = 0;
#pragma unroll
    for (int r = 0; r < kRows; r++) {
        cnt[r] = -1;
        if (r < rows) {
            const int i = base + 32 * r + lane;
            cnt[r] = cell_start[i + 1] - cell_start[i];
            mx = max(mx, cnt[r]);
        }
    }
    int v = __reduce_max_sync(FULL, mx);
    int pos = 0;  // lanes placed so far
    const unsigned below = (1u << lane) - 1u;
    while (v >= 0) {
        int next = -1;
#pragma unroll
        for (int r = 0; r < kRows; r++) {
            if (r >= rows) break;
            const bool mine = cnt[r] == v;
            const unsigned b = __ballot_sync(FULL, mine);
            if (mine) {
                const int l = pos + __popc(b & below), cell = 32 * r + lane;
                lane_cell[base + l] = base + cell;
                cell_lane[base + cell] = base + l;
                if ((l & 31) == 0) group_slots[(base + l) >> 5] = 32 * v;
            }
            pos += __popc(b);
            if (cnt[r] < v) next = max(next, cnt[r]);
        }
        v = __reduce_max_sync(FULL, next);
    }
}

// Slot of particle r of the cell with key k.
__device__ __forceinline__ int slot_in_cell(int k, int r, const int *cell_lane, const int *group_base)
{
    const int l = cell_lane[k];
    return group_base[l >> 5] + 32 * r + (l & 31);
}

// Slot of the particle at sorted position q (perm order = key order).
__device__ __forceinline__ int slot_of(int q, const int *perm, const int *key, const int *cell_start,
                                       const int *cell_lane, const int *group_base)
{
    const int k = key[perm[q]];
    return slot_in_cell(k, q - cell_start[k], cell_lane, group_base);
}

__device__ __forceinline__ uint32_t read_meta(const icy_SimParams &P, int i)
{
    const uint8_t *cr = (const uint8_t *)P.pts_array;
    const uint16_t *gr = (const uint16_t *)((const char *)P.pts_array + P.nPtsPitch);
    return (uint32_t)gr[i] | ((uint32_t)cr[i] << 16);
}

__global__ void k_pack64(const icy_SimParams P, const int *perm, const int *key, const int *cell_start,
                         const int *cell_lane, const int *group_base, int *pid, Parts64 A)
{
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= P.nPts) return;
    int i = perm[q];
    int k = slot_of(q, perm, key, cell_start, cell_lane, group_base);
    const double *pts = P.pts_array;
    const size_t pp = P.nPtsPitch;
    auto row = [&](int r) { return pts[(size_t)r * pp + i]; };
    pid[k] = i;
    A.pos[k] = make_double2(row(ICM_IDX_POSX), row(ICM_IDX_POSX + 1));
    A.vel[k] = make_double2(row(ICM_IDX_VELX), row(ICM_IDX_VELX + 1));
    A.F[k] = make_double4(row(ICM_IDX_FE00), row(ICM_IDX_FE00 + 1), row(ICM_IDX_FE00 + 2), row(ICM_IDX_FE00 + 3));
    A.Bp[k] = make_double4(row(ICM_IDX_BP00), row(ICM_IDX_BP00 + 1), row(ICM_IDX_BP00 + 2), row(ICM_IDX_BP00 + 3));
    A.Jp[k] = row(ICM_IDX_JP_INV);
    A.meta[k] = read_meta(P, i);
}

__global__ void k_unpack64(const icy_SimParams P, int nslots, const int *pid, const Parts64 A, int write_pq)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nslots) return;
    int i = pid[k];
    if (i < 0) return;
    double *pts = P.pts_array;
    const size_t pp = P.nPtsPitch;
    auto row = [&](int r) -> double & { return pts[(size_t)r * pp + i]; };
    double2 x = A.pos[k], v = A.vel[k];
    double4 F = A.F[k], B = A.Bp[k];
    row(ICM_IDX_POSX) = x.x; row(ICM_IDX_POSX + 1) = x.y;
    row(ICM_IDX_VELX) = v.x; row(ICM_IDX_VELX + 1) = v.y;
    row(ICM_IDX_FE00) = F.x; row(ICM_IDX_FE00 + 1) = F.y; row(ICM_IDX_FE00 + 2) = F.z; row(ICM_IDX_FE00 + 3) = F.w;
    row(ICM_IDX_BP00) = B.x; row(ICM_IDX_BP00 + 1) = B.y; row(ICM_IDX_BP00 + 2) = B.z; row(ICM_IDX_BP00 + 3) = B.w;
    row(ICM_IDX_JP_INV) = A.Jp[k];
    ((uint8_t *)pts)[i] = (uint8_t)(A.meta[k] >> 16);
    if (write_pq) {
        double2 q = A.pq[k];
        row(ICM_IDX_P) = q.x;
        row(ICM_IDX_Q) = q.y;
    }
}

__global__ void k_pack32(const icy_SimParams P, const int *perm, const int *key, const int *cell_start,
                         const int *cell_lane, const int *group_base, int *pid, Parts32 A)
{
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= P.nPts) return;
    int i = perm[q];
    int k = slot_of(q, perm, key, cell_start, cell_lane, group_base);
    const double *pts = P.pts_array;
    const size_t pp = P.nPtsPitch;
    auto row = [&](int r) { return pts[(size_t)r * pp + i]; };
    pid[k] = i;
    // cell and 32-bit fixed-point fraction of the position (a fraction that
    // rounds up to a whole cell carries into the cell)
    const double X = row(ICM_IDX_POSX) * P.cellsize_inv, Y = row(ICM_IDX_POSX + 1) * P.cellsize_inv;
    const double fx = floor(X), fy = floor(Y);
    long long ux = llrint((X - fx) * 4294967296.0), uy = llrint((Y - fy) * 4294967296.0);
    int ix = (int)fx, iy = (int)fy;
    if (ux >= 4294967296ll) { ux -= 4294967296ll; ix += 1; }
    if (uy >= 4294967296ll) { uy -= 4294967296ll; iy += 1; }
    const int16_t *gr = (const int16_t *)((const char *)P.pts_array + P.nPtsPitch);
    A.X[k] = pack_x32(ix, iy, (uint32_t)ux, (uint32_t)uy, grain_meta32(gr[i], ((const uint8_t *)P.pts_array)[i]));
    A.vel[k] = make_float2((float)row(ICM_IDX_VELX), (float)row(ICM_IDX_VELX + 1));
    A.H[k] = make_float4((float)(row(ICM_IDX_FE00) - 1.0), (float)row(ICM_IDX_FE00 + 1), (float)row(ICM_IDX_FE00 + 2),
                         (float)(row(ICM_IDX_FE00 + 3) - 1.0));
    A.Bp[k] = make_float4((float)row(ICM_IDX_BP00), (float)row(ICM_IDX_BP00 + 1), (float)row(ICM_IDX_BP00 + 2),
                          (float)row(ICM_IDX_BP00 + 3));
    A.Jp[k] = (float)(row(ICM_IDX_JP_INV) - 1.0);  // strain form
}

__global__ void k_unpack32(const icy_SimParams P, int nslots, const int *pid, const Parts32 A, int write_pq)
{
    int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nslots) return;
    int i = pid[k];
    if (i < 0) return;
    double *pts = P.pts_array;
    const size_t pp = P.nPtsPitch;
    auto row = [&](int r) -> double & { return pts[(size_t)r * pp + i]; };
    const float4 X = A.X[k];
    const uint32_t c = __float_as_uint(X.z);
    const float2 v = A.vel[k];
    float4 H = A.H[k], B = A.Bp[k];
    row(ICM_IDX_POSX) = ((double)cell_x(c) + (double)__float_as_uint(X.x) * 0x1p-32) * P.cellsize;
    row(ICM_IDX_POSX + 1) = ((double)cell_y(c) + (double)__float_as_uint(X.y) * 0x1p-32) * P.cellsize;
    row(ICM_IDX_VELX) = v.x; row(ICM_IDX_VELX + 1) = v.y;
    row(ICM_IDX_FE00) = 1.0 + (double)H.x; row(ICM_IDX_FE00 + 1) = H.y;
    row(ICM_IDX_FE00 + 2) = H.z; row(ICM_IDX_FE00 + 3) = 1.0 + (double)H.w;
    row(ICM_IDX_BP00) = B.x; row(ICM_IDX_BP00 + 1) = B.y; row(ICM_IDX_BP00 + 2) = B.z; row(ICM_IDX_BP00 + 3) = B.w;
    row(ICM_IDX_JP_INV) = 1.0 + (double)A.Jp[k];
    ((uint8_t *)pts)[i] = (uint8_t)meta32_crushed(__float_as_uint(X.w));
    if (write_pq) {
        float2 q = A.pq[k];
        row(ICM_IDX_P) = q.x;
        row(ICM_IDX_Q) = q.y;
    }
}

}  // namespace icm

// ------------------------------------------------------------- re-binning
//
// Particles drift out of the cell they were binned to; such "strays" take
// the per-particle scatter path. Between two steady-state launches the
// internal arrays are re-binned: keys from the current positions, a
// counting sort (deterministic inside a cell: particle order), new ELL slots
// and a gather into the spare arrays. Velocity and Bp are not part of the
// state between launches (the next G2P rebuilds them from the grid), and
// the scatter buffer of the next substep is already filled, so nothing else
// moves.

namespace icm {

__device__ __forceinline__ int key_of_base(const icy_SimParams &P, const TileGeom &g, int bx, int by)
{
    bx = min(max(bx, 0), P.GridX - 1);
    by = min(max(by, 0), P.GridY - 1);
    int tx = bx / g.TX, ty = by / g.TY;
    return ((ty * g.ntx + tx) * g.TY + (by - ty * g.TY)) * g.TX + (bx - tx * g.TX);
}

template <class Pol>
__global__ void k_rebin_keys(const icy_SimParams P, const typename Pol::Consts K, const TileGeom g, int nslots,
                             const int *pid, const typename Pol::Parts A, int *slot_key, int *count)
{
    int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= nslots || pid[slot] < 0) return;
    typename Pol::St s = Pol::load(A, slot);
    typename Pol::Sten st = Pol::stencil(P, K, s);
    int k = key_of_base(P, g, st.bx, st.by);
    slot_key[slot] = k;
    atomicAdd(&count[k], 1);
}

__global__ void k_rebin_scatter(int nslots, const int *pid, const int *slot_key, int *cursor, int *order)
{
    int slot = blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= nslots || pid[slot] < 0) return;
    int pos = atomicAdd(&cursor[slot_key[slot]], 1);
    order[pos] = slot;
}

// Insertion sort of each cell's slots by particle id (the atomic scatter
// order is not deterministic).
__global__ void k_rebin_order(int ncells, const int *start, int *order, const int *pid)
{
    int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= ncells) return;
    int a = start[c], b = start[c + 1];
    for (int i = a + 1; i < b; i++) {
        int v = order[i], pv = pid[v], j = i - 1;
        while (j >= a && pid[order[j]] > pv) { order[j + 1] = order[j]; j--; }
        order[j + 1] = v;
    }
}

__device__ __forceinline__ void copy_slot(const Parts32 &S, int from, const Parts32 &D, int to, bool pq)
{
    D.X[to] = S.X[from];
    D.H[to] = S.H[from];
    D.Jp[to] = S.Jp[from];
    if (pq) D.pq[to] = S.pq[from];
}
__device__ __forceinline__ void copy_slot(const Parts64 &S, int from, const Parts64 &D, int to, bool pq)
{
    D.pos[to] = S.pos[from];
    D.F[to] = S.F[from];
    D.Jp[to] = S.Jp[from];
    D.meta[to] = S.meta[from];
    if (pq) D.pq[to] = S.pq[from];
}

template <class Parts>
__global__ void k_rebin_gather(int n, const int *order, const int *slot_key, const int *cell_start,
                               const int *cell_lane, const int *group_base, const int *pid_old, int *pid_new,
                               const Parts S, const Parts D, int pq)
{
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    int old = order[q];
    int k = slot_key[old];
    int ns = slot_in_cell(k, q - cell_start[k], cell_lane, group_base);
    copy_slot(S, old, D, ns, pq != 0);
    pid_new[ns] = pid_old[old];
}

}  // namespace icm
