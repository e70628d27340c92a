// mpm_math32.cuh -- FP32 device math of the iceMPM substep in strain form.
//
// The FP32 form stores the elastic deformation gradient as H = Fe - I. Ice
// strains are ~1e-3, so Fe itself in FP32 would keep only ~4 significant
// digits of the strain; every quantity below is computed from H without
// forming 1 + small and subtracting 1 again.
//
// Invariants, shared by the Kirchhoff stress and the failure check:
//   J - 1 = tr H + det H,  b - I = F F^T - I = H + H^T + H H^T,
//   hd = ((b - I)_00 - (b - I)_11)/2,  b01 = (b - I)_01,
//   me = ((b - I)_00 + (b - I)_11)/2.
// Kirchhoff stress (gpu_implementation5.cu:24-34):
//   tau = s1 dev(b) + s2 I with s1 = mu/J, s2 = kappa (J^2 - 1).
// ComputePQ (gpu_implementation5.cu:36-44) needs no SVD for p and q: the
// squared singular values are the eigenvalues of b, so
//   p = -kappa/2 (J^2 - 1) = -s2/2,
//   q = sqrt(2) |mu/J dev(sigma^2)| = (mu/J)(sigma0^2 - sigma1^2)
//     = 2 s1 sqrt(hd^2 + b01^2).
// An intact particle whose (p, q) is clearly inside its failure surface is
// done here in FP32, and so is the Drucker-Prager map of a crushed particle
// (dp_map32: in strain form, from the same invariants, no SVD). The rest --
// the crush decision at the failure surface, a crushed particle within a
// relative 1e-4 of a discontinuity of the map, and ill-conditioned states
// (det F small or negative) -- is redone in FP64 with the reference form
// (mpm_math64.cuh).
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
    // Drucker-Prager map (Pa): threshold pressure, tan(phi), the
    // compressive and shear strengths it uses (not grain-varied), Je of the
    // hydrostatic reset sqrt(1 + 2 p_thr/kappa) and Je - 1
    float p_thr, tan_phi, dp_pmax, dp_qmax, je_new, je_new_m1;
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

// Stress and (p, q) of one H: J = det F, s1 = mu/J, s2 = kappa (J^2 - 1),
// and b - I = me I + [[hd, b01], [b01, -hd]] (eigenvalues me +- |(hd, b01)|,
// the squared singular values of F minus one).
struct Inv32 { float J, Jm1, s1, s2, hd, b01, me; };

__host__ __device__ __forceinline__ Inv32 invariants32(const M2f &H, float mu, float kappa)
{
    Inv32 v;
    v.Jm1 = (H.a00 + H.a11) + (H.a00 * H.a11 - H.a01 * H.a10);
    v.J = 1.0f + v.Jm1;
    float b00 = 2.0f * H.a00 + H.a00 * H.a00 + H.a01 * H.a01;
    float b11 = 2.0f * H.a11 + H.a10 * H.a10 + H.a11 * H.a11;
    v.b01 = H.a01 + H.a10 + H.a00 * H.a10 + H.a01 * H.a11;
    // (b00 - b11)/2 factored so that a mostly volumetric strain (b00 ~ b11)
    // does not cancel: (H00 - H11)(1 + (H00 + H11)/2) + (H01 - H10)(H01 + H10)/2
    v.hd = (H.a00 - H.a11) * (1.0f + 0.5f * (H.a00 + H.a11)) + 0.5f * (H.a01 - H.a10) * (H.a01 + H.a10);
    v.me = 0.5f * (b00 + b11);
#ifdef __CUDA_ARCH__
    v.s1 = __fdividef(mu, v.J);
#else
    v.s1 = mu / v.J;
#endif
    v.s2 = kappa * v.Jm1 * (v.J + 1.0f);
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

// Result codes of constitutive32 and dp_map32.
enum { kC32_OK = 0, kC32_NEEDS_FP64 = 1 };

// Relative distance from a discontinuity of the Drucker-Prager map (the
// hydrostatic threshold p = -p_thr, the compressive strength p = pmax)
// inside which the FP32 form redoes the map in FP64.
constexpr float kDpMargin = 1e-4f;

// Wolper_Drucker_Prager (gpu_implementation5.cu:48-94) of a crushed
// particle in strain form, without an SVD. With F = U S V^T and
// b = F F^T = U S^2 U^T, the map keeps U and V and replaces the singular
// values, so F_new = U diag(r) U^T F with r_i = s_new_i / s_i, and
//   H_new = F_new - I = (M - I) + (M - I) H + H,
//   M - I = U diag(r - 1) U^T = a I + c [[hd, b01], [b01, -hd]] / rho,
// a = (r0 - 1 + r1 - 1)/2, c = (r0 - r1)/2, rho = |(hd, b01)| (U's first
// column is b's eigenvector of the larger eigenvalue me + rho). Every term
// is formed from small quantities (strains), so FP32 keeps their relative
// accuracy:
// * hydrostatic branch (p < -p_thr or Jp_inv < 1): s_new_i^2 = Je_new, so
//   r_i^2 - 1 = (Je_new - 1 - e_i)/(1 + e_i) with e_i = me +- rho, and
//   Jp_inv *= Je_new / J, in strain form as the state keeps it (jpm1 =
//   Jp_inv - 1): with f - 1 = (Je_new - 1 - (J - 1)) / J, jpm1 += (f - 1) +
//   jpm1 (f - 1). (The factor rounded to float, 6e-8 relative, was enough to
//   move the 999,424-particle indentation to another crushing pattern within
//   10,000 substeps.)
// * cone (q >= q_n+1): the mean of s^2 is kept and its half-gap rho becomes
//   rho q_n+1 / q, so e_new_i - e_i = +-(rho_new - rho) and
//   r_i^2 - 1 = (e_new_i - e_i)/(1 + e_i);
// * inside the cone: unchanged.
// r_i - 1 = (r_i^2 - 1)/(sqrt(r_i^2) + 1) avoids the cancellation of
// sqrt(.) - 1. p and q are the trial state's (p = -s2/2, q = 2 s1 rho).
// Returns kC32_NEEDS_FP64 (state untouched) within kDpMargin of the map's
// discontinuities, where float rounding could select another branch than
// the FP64 form would.
// F_new = U diag(r) U^T F in strain form, given r_i - 1 (U: eigenvectors of
// b = F F^T, the first for the larger eigenvalue).
__host__ __device__ __forceinline__ void scale_principal32(M2f &H, const Inv32 &v, float rho, float r0m1, float r1m1)
{
    const float a = 0.5f * (r0m1 + r1m1), c = 0.5f * (r0m1 - r1m1);
    const float cn = rho > 0.0f ? c / rho : 0.0f;  // c = 0 whenever rho = 0
    const float m00 = a + cn * v.hd, m01 = cn * v.b01, m11 = a - cn * v.hd;
    const M2f h = H;
    H.a00 = h.a00 + (m00 + (m00 * h.a00 + m01 * h.a10));
    H.a01 = h.a01 + (m01 + (m00 * h.a01 + m01 * h.a11));
    H.a10 = h.a10 + (m01 + (m01 * h.a00 + m11 * h.a10));
    H.a11 = h.a11 + (m11 + (m01 * h.a01 + m11 * h.a11));
}

__host__ __device__ __forceinline__ int dp_map32(const Consts32 &k, M2f &H, float &jpm1, const Inv32 &v, float p,
                                                 float q, float rho)
{
    if (fabsf(p + k.p_thr) <= kDpMargin * fmaxf(k.p_thr, fabsf(p)) || fabsf(p - k.dp_pmax) <= kDpMargin * k.dp_pmax)
        return kC32_NEEDS_FP64;
    const float e0 = v.me + rho, e1 = v.me - rho;
    float d0, d1;  // r_i^2 - 1
    if (p < -k.p_thr || jpm1 < 0.0f) {
        d0 = (k.je_new_m1 - e0) / (1.0f + e0);
        d1 = (k.je_new_m1 - e1) / (1.0f + e1);
        const float fm1 = (k.je_new_m1 - v.Jm1) / v.J;
        jpm1 = jpm1 + (fm1 + jpm1 * fm1);
    } else {
        const float qn = (p > k.dp_pmax) ? 0.0f : fminf((p + k.p_thr) * k.tan_phi, k.dp_qmax);
        if (!(q >= qn) || !(q > 0.0f)) return kC32_OK;
        const float drho = -rho * ((q - qn) / q);  // rho_new - rho
        d0 = drho / (1.0f + e0);
        d1 = -drho / (1.0f + e1);
    }
    scale_principal32(H, v, rho, d0 / (sqrtf(1.0f + d0) + 1.0f), d1 / (sqrtf(1.0f + d1) + 1.0f));
    return kC32_OK;
}

// ComputePQ and dp_map32 of a crushed particle (kept out of line: crushed
// particles are few, and the map's values would add to the register
// pressure of every particle's update). tau is the Kirchhoff stress of the
// new H; rc is dp_map32's. jpm1 = Jp_inv - 1 (the state keeps Jp_inv in
// strain form).
struct Crushed32 { M2f H; float jpm1, p, q; Tau32 tau; int rc; };

static __device__ __noinline__ Crushed32 crushed32(const Consts32 &k, const M2f H, const float jpm1)
{
    Crushed32 o{H, jpm1, 0.0f, 0.0f, {0.0f, 0.0f, 0.0f}, kC32_OK};
    const Inv32 v = invariants32(H, k.mu, k.kappa);
    const float rho = sqrtf(v.hd * v.hd + v.b01 * v.b01);
    o.p = -0.5f * v.s2;
    o.q = 2.0f * v.s1 * rho;
    o.rc = dp_map32(k, o.H, o.jpm1, v, o.p, o.q, rho);
    if (o.rc == kC32_OK) o.tau = tau32(invariants32(o.H, k.mu, k.kappa));
    return o;
}

// ComputePQ, then for an intact particle the failure check, for a crushed
// one the Drucker-Prager map (dp_map32); tau is the Kirchhoff stress of the
// new H. Returns kC32_NEEDS_FP64 (state untouched) for an intact particle on
// or outside its failure surface or within kSurfaceMargin of it, for a
// crushed one near a discontinuity of the map, and for det F <= 0.25.
// jpm1 = Jp_inv - 1.
__device__ __forceinline__ int constitutive32(const Consts32 &k, const GrainTables32 &T, M2f &H, float &jpm1,
                                              uint32_t meta, float &p_tr, float &q_tr, Tau32 &tau)
{
    Inv32 v = invariants32(H, k.mu, k.kappa);
    if (!(v.J > 0.25f)) return kC32_NEEDS_FP64;
    const float p = -0.5f * v.s2;
    if (meta32_crushed(meta)) {
        const Crushed32 o = crushed32(k, H, jpm1);
        if (o.rc != kC32_OK) return kC32_NEEDS_FP64;
        H = o.H;
        jpm1 = o.jpm1;
        p_tr = o.p;
        q_tr = o.q;
        tau = o.tau;
        return kC32_OK;
    }
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
// loop. jpm1 = Jp_inv - 1 in and out.
struct Via64 { M2f H; float jpm1, p_tr, q_tr; uint32_t meta; };

static __device__ __noinline__ Via64 constitutive32_via64(const icy_SimParams &P, const M2f H, const float jpm1,
                                                          const uint32_t meta)
{
    M2d F = {1.0 + (double)H.a00, (double)H.a01, (double)H.a10, 1.0 + (double)H.a11};
    double jp = 1.0 + (double)jpm1, p, q;
    uint8_t cr = (uint8_t)meta32_crushed(meta);
    constitutive64(P, F, jp, cr, meta32_res(meta), p, q);
    Via64 o;
    o.H = {(float)(F.a00 - 1.0), (float)F.a01, (float)F.a10, (float)(F.a11 - 1.0)};
    o.jpm1 = (float)(jp - 1.0);
    o.p_tr = (float)p;
    o.q_tr = (float)q;
    o.meta = (meta & 0x00ffffffu) | ((uint32_t)cr << 24);
    return o;
}

}  // namespace icm
