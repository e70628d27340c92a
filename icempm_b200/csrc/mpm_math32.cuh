// mpm_math32.cuh -- FP32 device math of the iceMPM substep in strain form.
//
// The FP32 form stores the elastic deformation gradient as H = Fe - I. Ice
// strains are ~1e-3, so Fe itself in FP32 would keep only ~4 significant
// digits of the strain; every quantity below is computed from H without
// forming 1 + small and subtracting 1 again.
//
// Invariants, shared by the Kirchhoff stress and the failure check:
//   J - 1 = tr H + det H,  b - I = F F^T - I = H + H^T + H H^T,
//   hd = ((b - I)_00 - (b - I)_11)/2,  b01 = (b - I)_01.
// Kirchhoff stress (gpu_implementation5.cu:24-34):
//   tau = s1 dev(b) + s2 I with s1 = mu/J, s2 = kappa (J^2 - 1).
// ComputePQ (gpu_implementation5.cu:36-44) needs no SVD for p and q: the
// squared singular values are the eigenvalues of b, so
//   p = -kappa/2 (J^2 - 1) = -s2/2,
//   q = sqrt(2) |mu/J dev(sigma^2)| = (mu/J)(sigma0^2 - sigma1^2)
//     = 2 s1 sqrt(hd^2 + b01^2).
// An intact particle whose (p, q) is clearly inside its failure surface is
// done here in FP32. Everything else -- the crush decision at the surface,
// every crushed particle (SVD + Drucker-Prager map, gpu_implementation5.cu:
// 48-94, helper_math.cuh:27-140) and ill-conditioned states (det F small or
// negative) -- is redone in FP64 with the reference form (mpm_math64.cuh).
// Crushed particles are a fraction of a percent of a block and sit together
// near the indenter, so this costs no measurable time; it is done for all of
// them, not only for nearly equal singular values, because the indentation's
// crushing outcome is sensitive to strain perturbations of a few 1e-8 and an
// FP32 return map moved the peak indenter force of a 10k-substep run by ~4%.
#pragma once
#include <cstdint>
#include "mpm_math64.cuh"

namespace icm {

struct M2f { float a00, a01, a10, a11; };
struct MlpWarpNet;

// Per-run FP32 constants, derived on the host in double.
struct Consts32 {
    float h, h_inv, dt, dt_h_inv, mass, stress_c;  // stress_c = dt*Vp*Dinv
    float mu, kappa;
    float gv, ics, its, iss;                        // grain variability, strengths in MPa
    float four_h_inv;
    float dt_g, vmax;                               // dt*gravity, 0.5 h/dt
    // a box in (p, q) (MPa) inside every failure surface that a grain with a
    // non-negative id can have, with a wide margin: a particle of such a
    // grain inside it needs no table lookup to be found intact (q2 = 0: none)
    float inside_plo, inside_phi, inside_q2;
    // trial states of crushed particles (H, Jp_inv, meta: 6 words each) are
    // appended here while harvest is set (training data of the surrogate)
    float *harvest;
    unsigned *harvest_n;
    unsigned harvest_cap;
    // surrogate form: network, acceptance tolerance, counters {accepted, exact}
    const MlpWarpNet *mlp;
    float mlp_tol;
    unsigned long long *mlp_counts;
};

// Grain strengths in MPa by residue (gpu_implementation5.cu:97-105): the
// grain id enters only through grain % 21, (grain + 3) % 30 and
// (grain + 4) % 11, stored per particle at pack time offset by +20, +29,
// +10 so that negative ids stay in range.
struct GrainTables32 { float pmax[41], pmin[59], qmax[21]; };

__device__ __forceinline__ void grain_tables32_init(GrainTables32 &T, const Consts32 &k, int tid, int nthr)
{
    for (int r = tid; r < 41 + 59 + 21; r += nthr) {
        if (r < 41) T.pmax[r] = k.ics * (1.0f + k.gv * 0.05f * (float)(-10 + (r - 20)));
        else if (r < 100) T.pmin[r - 41] = -k.its * (1.0f + k.gv * 0.033f * (float)(-15 + (r - 41 - 29)));
        else T.qmax[r - 100] = k.iss * (1.0f + k.gv * 0.1f * (float)(-10 + (r - 100 - 10)));
    }
}

// meta word of the FP32 form: residues in bits 0-5, 6-11, 12-16; crushed
// flag in bits 24-31.
__host__ __device__ __forceinline__ uint32_t grain_meta32(int grain, int crushed)
{
    uint32_t r1 = (uint32_t)(grain % 21 + 20), r2 = (uint32_t)((grain + 3) % 30 + 29), r3 = (uint32_t)((grain + 4) % 11 + 10);
    return r1 | (r2 << 6) | (r3 << 12) | ((uint32_t)crushed << 24);
}
__device__ __forceinline__ int meta32_crushed(uint32_t m) { return (int)(m >> 24); }

// The reference's grain remainders (grain_res) of a meta word.
__device__ __forceinline__ GrainRes meta32_res(uint32_t m)
{
    return {(int)(m & 63u) - 20, (int)((m >> 6) & 63u) - 29, (int)((m >> 12) & 31u) - 10};
}

// Stress and (p, q) of one H.
struct Inv32 { float J, s1, s2, hd, b01; };

__device__ __forceinline__ Inv32 invariants32(const M2f &H, float mu, float kappa)
{
    Inv32 v;
    float Jm1 = (H.a00 + H.a11) + (H.a00 * H.a11 - H.a01 * H.a10);
    v.J = 1.0f + Jm1;
    float b00 = 2.0f * H.a00 + H.a00 * H.a00 + H.a01 * H.a01;
    float b11 = 2.0f * H.a11 + H.a10 * H.a10 + H.a11 * H.a11;
    v.b01 = H.a01 + H.a10 + H.a00 * H.a10 + H.a01 * H.a11;
    v.hd = 0.5f * (b00 - b11);
    v.s1 = __fdividef(mu, v.J);
    v.s2 = kappa * Jm1 * (v.J + 1.0f);
    return v;
}

// tau = s1 dev(b) + s2 I as {t00, t01, t11} (symmetric)
struct Tau32 { float t00, t01, t11; };
__device__ __forceinline__ Tau32 tau32(const Inv32 &v) { return {v.s1 * v.hd + v.s2, v.s1 * v.b01, -v.s1 * v.hd + v.s2}; }

__device__ __forceinline__ float approx_sqrt(float x) { return x > 0.0f ? x * rsqrtf(x) : 0.0f; }

// Grain-varied failure surface (gpu_implementation5.cu:97-141) in FP32,
// rearranged without divisions and in MPa so every product stays in range:
//   p < 0:  crushed if p < -3 MPa, or if q > q0 (p + 3 MPa)/(3 MPa) with
//           q0 = 2 sqrt(-pmax pmin) qmax/(pmax - pmin), i.e.
//           9 q^2 (pmax - pmin)^2 > 4 (-pmax pmin) qmax^2 (p + 3)^2;
//   p >= 0: y = (1 + 2 beta) q^2 + M^2 (p + beta pmax)(p - pmax) > 0 with
//           beta = -pmin/pmax and M^2 = 4 qmax^2 (1 + 2 beta)/(pmax (1 + beta))^2
//           has the sign of q^2 (pmax - pmin)^2 + 4 qmax^2 (p - pmin)(p - pmax)
//           (1 + 2 beta > 0 and pmax (1 + beta) = pmax - pmin).
// Returns 1 (outside), 0 (inside) or -1 when the point lies within a
// relative margin of the surface, where the FP32 decision is not trusted.
constexpr float kSurfaceMargin = 1e-3f;

__device__ __forceinline__ int failure_side32(const GrainTables32 &T, uint32_t meta, float p_pa, float q_pa)
{
    float pmax = T.pmax[meta & 63u];
    float pmin = T.pmin[(meta >> 6) & 63u];
    float qmax = T.qmax[(meta >> 12) & 31u];
    float p = p_pa * 1e-6f, q = q_pa * 1e-6f;
    float dpm = pmax - pmin;
    // Both branches have the same sign at p = 0; at p = -3 MPa only q ~ 0 is ambiguous.
    if (fabsf(p + 3.0f) < 3.0f * kSurfaceMargin) return -1;
    if (p < 0.0f) {
        if (p < -3.0f) return 1;
        float l = 3.0f * q * dpm, r2 = 4.0f * (-pmax * pmin) * qmax * qmax;
        float pp = p + 3.0f;
        float a = l * l, b = r2 * pp * pp;
        if (fabsf(a - b) <= 2.0f * kSurfaceMargin * (a + b)) return -1;
        return a > b ? 1 : 0;
    }
    float a = q * q * dpm * dpm, b = 4.0f * qmax * qmax * (p - pmin) * (p - pmax);
    if (fabsf(a + b) <= kSurfaceMargin * (a + fabsf(b))) return -1;
    return a + b > 0.0f ? 1 : 0;
}

// Result codes of constitutive32.
enum { kC32_OK = 0, kC32_NEEDS_FP64 = 1 };

// ComputePQ + failure check of an intact particle whose (p, q) lies clearly
// inside its failure surface: the state is unchanged, tau is the Kirchhoff
// stress of H. Returns kC32_NEEDS_FP64 (state untouched) for a crushed
// particle, for one on or outside the surface or within kSurfaceMargin of
// it, and for det F <= 0.25.
__device__ __forceinline__ int constitutive32(const Consts32 &k, const GrainTables32 &T, const M2f &H, uint32_t meta,
                                              float &p_tr, float &q_tr, Tau32 &tau)
{
    Inv32 v = invariants32(H, k.mu, k.kappa);
    if (!(v.J > 0.25f) || meta32_crushed(meta)) return kC32_NEEDS_FP64;
    float p = -0.5f * v.s2;
    float q = 2.0f * v.s1 * approx_sqrt(v.hd * v.hd + v.b01 * v.b01);
    // residues at or above their offsets: the grain id is not negative
    const bool grain_nonneg = (meta & 63u) >= 20u && ((meta >> 6) & 63u) >= 29u && ((meta >> 12) & 31u) >= 10u;
    const float pm = p * 1e-6f, qm = q * 1e-6f;
    const bool clearly_inside = grain_nonneg && pm > k.inside_plo && pm < k.inside_phi && qm * qm < k.inside_q2;
    if (!clearly_inside && failure_side32(T, meta, p, q) != 0) return kC32_NEEDS_FP64;
    p_tr = p;
    q_tr = q;
    tau = tau32(v);
    return kC32_OK;
}

// FP64 redo of one particle for the cases constitutive32 declines (kept out
// of line). Takes and returns values: state passed by reference to an
// out-of-line call would have to live in local memory in the caller's hot
// loop.
struct Via64 { M2f H; float Jp, p_tr, q_tr; uint32_t meta; };

__device__ __noinline__ Via64 constitutive32_via64(const icy_SimParams &P, const M2f H, const float Jp_inv,
                                                   const uint32_t meta)
{
    M2d F = {1.0 + (double)H.a00, (double)H.a01, (double)H.a10, 1.0 + (double)H.a11};
    double jp = Jp_inv, p, q;
    uint8_t cr = (uint8_t)meta32_crushed(meta);
    constitutive64(P, F, jp, cr, meta32_res(meta), p, q);
    Via64 o;
    o.H = {(float)(F.a00 - 1.0), (float)F.a01, (float)F.a10, (float)(F.a11 - 1.0)};
    o.Jp = (float)jp;
    o.p_tr = (float)p;
    o.q_tr = (float)q;
    o.meta = (meta & 0x00ffffffu) | ((uint32_t)cr << 24);
    return o;
}

}  // namespace icm
