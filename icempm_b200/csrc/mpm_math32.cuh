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
// Only a crushed particle needs U and V (the Drucker-Prager map rebuilds Fe
// from them, gpu_implementation5.cu:48-94); its SVD follows the reference's
// route (polar decomposition, then a symmetric eigen-solve,
// helper_math.cuh:27-46,81-140) in strain form: F = R S, S = I + E with E
// from H and cos(theta) - 1 = -b^2/(d(a+d)); sigma_i = 1 + e_i. The
// projected stretches enter as delta_i = sigma_new_i - 1 =
// (B_i - 1)/(sqrt(B_i) + 1) and H_new = R V diag(delta) V^T + (R - I).
// Where this is ill-conditioned -- det F small or negative, a large rotation
// (tr F <= 0.5), large strain, or nearly equal singular values of a crushed
// particle -- the caller redoes the particle in FP64 with the reference form
// (mpm_math64.cuh).
#pragma once
#include <cstdint>
#include "mpm_math64.cuh"

namespace icm {

struct M2f { float a00, a01, a10, a11; };

// Per-run FP32 constants, derived on the host in double.
struct Consts32 {
    float h, h_inv, dt, dt_h_inv, mass, stress_c;  // stress_c = dt*Vp*Dinv
    float mu, kappa, tan_phi, p_thr, pmax_dp, qmax_dp;
    float tension_Je_new, tension_delta;            // sqrt(1 + 2 p_thr/kappa), sqrt(Je_new) - 1
    float gv, ics, its, iss;                        // grain variability, strengths in MPa
    float four_h_inv;
    float dt_g, vmax, half_inv_mu;                  // dt*gravity, 0.5 h/dt, 1/(2 mu)
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

// A grain id with the same residues (for the FP64 redo, which evaluates
// GetParametersForGrain): ids with equal grain % 21, (grain + 3) % 30 and
// (grain + 4) % 11 have equal parameters; the residues repeat with period
// 2310, searched only on that rare path.
__device__ __forceinline__ int meta32_grain(uint32_t m)
{
    int r1 = (int)(m & 63u) - 20, r2 = (int)((m >> 6) & 63u) - 29, r3 = (int)((m >> 12) & 31u) - 10;
    int base = (r1 < 0 || r2 < 0 || r3 < 0) ? -2309 : 0;
    for (int g = base; g < base + 2310; g++)
        if (g % 21 == r1 && (g + 3) % 30 == r2 && (g + 4) % 11 == r3) return g;
    return 0;
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

struct Svd32 {
    float c, s;    // R = [[c, -s], [s, c]]
    float cm1;     // c - 1, computed without cancellation
    float vc, vs;  // V = [[vc, -vs], [vs, vc]]: columns are the eigenvectors of S
    float e0, e1;  // sigma_i - 1, e0 >= e1
    float w;       // (e0 - e1)/2
    float a;       // tr F, the polar denominator's first component
};

__device__ __forceinline__ Svd32 svd_strain32(const M2f &H)
{
    Svd32 r;
    float a = 2.0f + H.a00 + H.a11;
    float b = H.a10 - H.a01;
    r.a = a;
    float d = sqrtf(a * a + b * b);
    float inv_d = 1.0f / d;
    r.c = a * inv_d;
    r.s = b * inv_d;
    r.cm1 = __fdividef(-(b * b) * inv_d, a + d);
    float E00 = r.cm1 + r.c * H.a00 + r.s * H.a10;
    float E11 = r.cm1 - r.s * H.a01 + r.c * H.a11;
    float E01 = r.s + r.c * H.a01 + r.s * H.a11;
    float E10 = -r.s - r.s * H.a00 + r.c * H.a10;
    float y = 0.5f * (E01 + E10);
    float mean = 0.5f * (E00 + E11);
    float tau = 0.5f * (E00 - E11);
    float w = sqrtf(tau * tau + y * y);
    r.w = w;
    r.e0 = mean + w;
    r.e1 = mean - w;
    // eigenvector of the larger eigenvalue, from the better-conditioned row
    float vx, vy;
    if (tau >= 0.0f) {
        vx = w + tau;
        vy = y;
    } else {
        vx = y;
        vy = w - tau;
    }
    float n2 = vx * vx + vy * vy;
    if (n2 > 0.0f) {
        float inv = rsqrtf(n2);
        r.vc = vx * inv;
        r.vs = vy * inv;
    } else {
        r.vc = 1.0f;
        r.vs = 0.0f;
    }
    return r;
}

// Grain-varied failure surface (gpu_implementation5.cu:97-141) in FP32,
// rearranged without divisions and in MPa so every product stays in range:
//   p < 0:  crushed if p < -3 MPa, or if q > q0 (p + 3 MPa)/(3 MPa) with
//           q0 = 2 sqrt(-pmax pmin) qmax/(pmax - pmin), i.e.
//           9 q^2 (pmax - pmin)^2 > 4 (-pmax pmin) qmax^2 (p + 3)^2;
//   p >= 0: y = (1 + 2 beta) q^2 + M^2 (p + beta pmax)(p - pmax) > 0 with
//           beta = -pmin/pmax and M^2 = 4 qmax^2 (1 + 2 beta)/(pmax (1 + beta))^2
//           has the sign of q^2 (pmax - pmin)^2 + 4 qmax^2 (p - pmin)(p - pmax)
//           (1 + 2 beta > 0 and pmax (1 + beta) = pmax - pmin).
__device__ __forceinline__ bool outside_failure_surface32(const GrainTables32 &T, uint32_t meta, float p_pa,
                                                          float q_pa)
{
    float pmax = T.pmax[meta & 63u];
    float pmin = T.pmin[(meta >> 6) & 63u];
    float qmax = T.qmax[(meta >> 12) & 31u];
    float p = p_pa * 1e-6f, q = q_pa * 1e-6f;
    float dpm = pmax - pmin;
    if (p < 0.0f) {
        if (p < -3.0f) return true;
        float l = 3.0f * q * dpm, r2 = 4.0f * (-pmax * pmin) * qmax * qmax;
        float pp = p + 3.0f;
        return l * l > r2 * pp * pp;
    }
    return q * q * dpm * dpm + 4.0f * qmax * qmax * (p - pmin) * (p - pmax) > 0.0f;
}

// Result codes of constitutive32.
enum { kC32_OK = 0, kC32_NEEDS_FP64 = 1 };

// ComputePQ + failure check + DP map on H (already advected). On return
// tau holds the Kirchhoff stress of the final H. Returns kC32_NEEDS_FP64
// without touching the state when the FP32 form is ill-conditioned.
__device__ __forceinline__ int constitutive32(const Consts32 &k, const GrainTables32 &T, M2f &H, float &Jp_inv,
                                              uint32_t &meta, float &p_tr, float &q_tr, Tau32 &tau)
{
    Inv32 v = invariants32(H, k.mu, k.kappa);
    if (!(v.J > 0.25f)) return kC32_NEEDS_FP64;
    float rad = approx_sqrt(v.hd * v.hd + v.b01 * v.b01);
    float p = -0.5f * v.s2;
    float q = 2.0f * v.s1 * rad;
    uint32_t m = meta;
    if (meta32_crushed(m) == 0 && outside_failure_surface32(T, m, p, q)) m |= 1u << 24;
    if (meta32_crushed(m)) {
        Svd32 d = svd_strain32(H);
        if (!(d.a > 0.5f) || !(d.e1 > -0.5f) || !(d.e0 < 1.0f)) return kC32_NEEDS_FP64;
        float scale = fabsf(d.e0) + fabsf(d.e1);
        if (d.w > 0.0f && d.w < 1e-5f * scale) return kC32_NEEDS_FP64;  // nearly equal stretches
        float d0, d1;
        bool change = true;
        if (p < -k.p_thr || Jp_inv < 1.0f) {
            d0 = d1 = k.tension_delta;
            Jp_inv *= __fdividef(k.tension_Je_new, v.J);
        } else {
            float q_n_1 = (p > k.pmax_dp) ? 0.0f : fminf((p + k.p_thr) * k.tan_phi, k.qmax_dp);
            if (q >= q_n_1) {
                float m1 = 0.5f * (d.e0 * (2.0f + d.e0) + d.e1 * (2.0f + d.e1));  // mean(sigma^2) - 1
                float g = (rad > 0.0f) ? q_n_1 * v.J * k.half_inv_mu : 0.0f;
                float B0 = m1 + g, B1 = m1 - g;  // B_i - 1
                d0 = __fdividef(B0, approx_sqrt(1.0f + B0) + 1.0f);
                d1 = __fdividef(B1, approx_sqrt(1.0f + B1) + 1.0f);
            } else {
                change = false;
            }
        }
        if (change) {
            // W = V diag(d0, d1) V^T; H = R W + (R - I)
            float cc = d.vc * d.vc, ss = d.vs * d.vs, cs = d.vc * d.vs;
            float W00 = d0 * cc + d1 * ss;
            float W11 = d0 * ss + d1 * cc;
            float W01 = (d0 - d1) * cs;
            H.a00 = d.c * W00 - d.s * W01 + d.cm1;
            H.a01 = d.c * W01 - d.s * W11 - d.s;
            H.a10 = d.s * W00 + d.c * W01 + d.s;
            H.a11 = d.s * W01 + d.c * W11 + d.cm1;
            v = invariants32(H, k.mu, k.kappa);
        }
    }
    meta = m;
    p_tr = p;
    q_tr = q;
    tau = tau32(v);
    return kC32_OK;
}

// FP64 redo of one particle for the cases constitutive32 declines (rare; kept
// out of line).
__device__ __noinline__ void constitutive32_via64(const icy_SimParams &P, M2f &H, float &Jp_inv, uint32_t &meta,
                                                  float &p_tr, float &q_tr)
{
    M2d F = {1.0 + (double)H.a00, (double)H.a01, (double)H.a10, 1.0 + (double)H.a11};
    double jp = Jp_inv, p, q;
    uint8_t cr = (uint8_t)meta32_crushed(meta);
    constitutive64(P, F, jp, cr, meta32_grain(meta), p, q);
    H = {(float)(F.a00 - 1.0), (float)F.a01, (float)F.a10, (float)(F.a11 - 1.0)};
    Jp_inv = (float)jp;
    p_tr = (float)p;
    q_tr = (float)q;
    meta = (meta & 0x00ffffffu) | ((uint32_t)cr << 24);
}

}  // namespace icm
