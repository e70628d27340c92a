// mpm_math32.cuh -- FP32 device math of the iceMPM substep in strain form.
//
// The FP32 form stores the elastic deformation gradient as H = Fe - I. Ice
// strains are ~1e-3, so Fe itself in FP32 would keep only ~4 significant
// digits of the strain; every quantity below is computed from H without
// forming 1 + small and subtracting 1 again:
//   Kirchhoff stress (gpu_implementation5.cu:24-34):
//     J - 1 = tr H + det H,  dev(F F^T) = dev(H + H^T + H H^T)
//   SVD (helper_math.cuh:27-46,81-140, same polar + symmetric eigen route):
//     F = R S, S = I + E with E computed from H and cos(theta) - 1 = -b^2/(d(a+d)),
//     sigma_i = 1 + e_i from the eigenvalues e_i of E.
//   p, q (gpu_implementation5.cu:36-44): J - 1 = tr H + det H,
//     sigma0^2 - sigma1^2 = (e0 - e1)(2 + e0 + e1).
//   Drucker-Prager (gpu_implementation5.cu:48-94): the projected stretches
//     enter as delta_i = sigma_new_i - 1 = (B_i - 1)/(sqrt(B_i) + 1) and
//     H_new = R V diag(delta) V^T + (R - I).
//   Failure check (gpu_implementation5.cu:97-141) in FP32 on (p, q).
// Where this is ill-conditioned -- a large rotation or inversion (a <= 0.5),
// large strain, or nearly equal singular values of a crushed particle -- the
// caller redoes the particle in FP64 with the reference form (mpm_math64.cuh).
#pragma once
#include <cstdint>
#include "mpm_math64.cuh"

namespace icm {

struct M2f { float a00, a01, a10, a11; };

// Per-run FP32 constants, derived on the host in double.
struct Consts32 {
    float h, h_inv, dt, dt_h_inv, mass, stress_c;  // stress_c = dt*Vp*Dinv
    float mu, kappa, half_kappa, tan_phi, p_thr, pmax_dp, qmax_dp;
    float tension_Je_new, tension_delta;            // sqrt(1 + 2 p_thr/kappa), sqrt(Je_new) - 1
    float gv, ics, its, iss;                        // grain variability, strengths
    float four_h_inv;
};

// tau = mu/J dev(F F^T) + kappa (J^2 - 1) I with F = I + H.
__device__ __forceinline__ M2f kirchhoff32(const M2f &H, float mu, float kappa)
{
    float Jm1 = (H.a00 + H.a11) + (H.a00 * H.a11 - H.a01 * H.a10);
    float J = 1.0f + Jm1;
    float b00 = 2.0f * H.a00 + H.a00 * H.a00 + H.a01 * H.a01;
    float b11 = 2.0f * H.a11 + H.a10 * H.a10 + H.a11 * H.a11;
    float b01 = H.a01 + H.a10 + H.a00 * H.a10 + H.a01 * H.a11;
    float hd = 0.5f * (b00 - b11);
    float s1 = mu / J;
    float s2 = kappa * Jm1 * (J + 1.0f);
    return {s1 * hd + s2, s1 * b01, s1 * b01, -s1 * hd + s2};
}

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
    r.cm1 = -(b * b) * inv_d / (a + d);
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

// Grain-varied failure surface (gpu_implementation5.cu:97-141) in FP32.
__device__ __forceinline__ bool outside_failure_surface32(const Consts32 &k, int grain, float p, float q)
{
    float var1 = 1.0f + k.gv * 0.05f * (float)(-10 + grain % 21);
    float var2 = 1.0f + k.gv * 0.033f * (float)(-15 + (grain + 3) % 30);
    float var3 = 1.0f + k.gv * 0.1f * (float)(-10 + (grain + 4) % 11);
    float pmax = k.ics * var1;
    float pmin = -k.its * var2;
    float qmax = k.iss * var3;
    float beta = -pmin / pmax;
    const float pmin2 = -3e6f;
    if (p < 0.0f) {
        if (p < pmin2) return true;
        float q0 = 2.0f * sqrtf(-pmax * pmin) * qmax / (pmax - pmin);
        float kk = -q0 / pmin2;
        return q > kk * (p - pmin2);
    }
    float t = pmax * (1.0f + beta);
    float mSq = (4.0f * qmax * qmax * (1.0f + 2.0f * beta)) / (t * t);
    float yv = (1.0f + 2.0f * beta) * q * q + mSq * (p + beta * pmax) * (p - pmax);
    return yv > 0.0f;
}

// Result codes of constitutive32.
enum { kC32_OK = 0, kC32_NEEDS_FP64 = 1 };

// ComputePQ + failure check + DP map on H (already advected). Returns
// kC32_NEEDS_FP64 without touching the state when the FP32 form is
// ill-conditioned for this particle.
__device__ __forceinline__ int constitutive32(const Consts32 &k, M2f &H, float &Jp_inv, uint8_t &crushed,
                                              int grain, float &p_tr, float &q_tr)
{
    Svd32 d = svd_strain32(H);
    if (!(d.a > 0.5f) || !(d.e1 > -0.5f) || !(d.e0 < 1.0f)) return kC32_NEEDS_FP64;
    // J - 1 = det(I + H) - 1 = tr H + det H: exact algebra, no cancellation
    // between the eigenvalues under pure shear
    float Jm1 = (H.a00 + H.a11) + (H.a00 * H.a11 - H.a01 * H.a10);
    float Je = 1.0f + Jm1;
    float p = -k.half_kappa * Jm1 * (Je + 1.0f);
    float D = 2.0f * d.w * (2.0f + d.e0 + d.e1);  // sigma0^2 - sigma1^2 >= 0
    float q = k.mu * D / Je;
    uint8_t cr = crushed;
    if (cr == 0 && outside_failure_surface32(k, grain, p, q)) cr = 1;
    if (cr == 1) {
        float scale = fabsf(d.e0) + fabsf(d.e1);
        if (d.w > 0.0f && d.w < 1e-5f * scale) return kC32_NEEDS_FP64;  // nearly equal stretches
        float d0, d1;
        bool change = true;
        if (p < -k.p_thr || Jp_inv < 1.0f) {
            d0 = d1 = k.tension_delta;
            Jp_inv *= k.tension_Je_new / Je;
        } else {
            float q_n_1 = (p > k.pmax_dp) ? 0.0f : fminf((p + k.p_thr) * k.tan_phi, k.qmax_dp);
            if (q >= q_n_1) {
                float m1 = 0.5f * (d.e0 * (2.0f + d.e0) + d.e1 * (2.0f + d.e1));  // mean(sigma^2) - 1
                float g = (D > 0.0f) ? q_n_1 * Je / (2.0f * k.mu) : 0.0f;
                float B0 = m1 + g, B1 = m1 - g;  // B_i - 1
                d0 = B0 / (sqrtf(1.0f + B0) + 1.0f);
                d1 = B1 / (sqrtf(1.0f + B1) + 1.0f);
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
        }
    }
    crushed = cr;
    p_tr = p;
    q_tr = q;
    return kC32_OK;
}

// FP64 redo of one particle for the cases constitutive32 declines.
__device__ __forceinline__ void constitutive32_via64(const icy_SimParams &P, M2f &H, float &Jp_inv,
                                                     uint8_t &crushed, int grain, float &p_tr, float &q_tr)
{
    M2d F = {1.0 + (double)H.a00, (double)H.a01, (double)H.a10, 1.0 + (double)H.a11};
    double jp = Jp_inv, p, q;
    constitutive64(P, F, jp, crushed, grain, p, q);
    H = {(float)(F.a00 - 1.0), (float)F.a01, (float)F.a10, (float)(F.a11 - 1.0)};
    Jp_inv = (float)jp;
    p_tr = (float)p;
    q_tr = (float)q;
}

}  // namespace icm
