// mpm_math64.cuh -- FP64 device math of the iceMPM substep, reference form.
//
// Register-only restatements of the reference device functions (paths inside
// the iceMPM project):
//   KirchhoffStress_Wolper        simulation/gpu_implementation5.cu:24-34
//   ComputePQ                     simulation/gpu_implementation5.cu:36-44
//   Wolper_Drucker_Prager         simulation/gpu_implementation5.cu:48-94
//   GetParametersForGrain         simulation/gpu_implementation5.cu:97-111
//   CheckIfPointIsInsideFailure.. simulation/gpu_implementation5.cu:114-141
//   svd / svd2x2_modified         simulation/gpu_implementation5.cu:399-416
//   polar + symmetric eigen SVD   simulation/helper_math.cuh:27-46,81-140
//   Givens rotation algebra       simulation/givens.cuh:100-128,161-166
// The 2x2 SVD keeps the reference's conventions: sigma0 >= sigma1, sigma1
// may be negative, U and V are rotations with F = U diag(sigma) V^T.
// Matrices are row-major {a00, a01, a10, a11}.
#pragma once
#include <cstdint>
#include "../../include/icempm_params.h"

namespace icm {

struct M2d { double a00, a01, a10, a11; };

constexpr double kCoeff1 = 1.4142135623730950;  // sqrt((6-d)/2), d = 2

__host__ __device__ __forceinline__ double det(const M2d &F) { return F.a00 * F.a11 - F.a10 * F.a01; }

// Kirchhoff stress tau = mu/J dev(F F^T) + kappa (J^2 - 1) I.
__device__ __forceinline__ M2d kirchhoff64(const M2d &F, double mu, double kappa)
{
    double Je = det(F);
    double b00 = F.a00 * F.a00 + F.a01 * F.a01;
    double b01 = F.a00 * F.a10 + F.a01 * F.a11;
    double b10 = F.a10 * F.a00 + F.a11 * F.a01;
    double b11 = F.a10 * F.a10 + F.a11 * F.a11;
    double half_tr = (b00 + b11) / 2;
    double s1 = mu * (1 / Je);
    double s2 = kappa * (Je * Je - 1.);
    return {s1 * (b00 - half_tr) + s2, s1 * b01, s1 * b10, s1 * (b11 - half_tr) + s2};
}

// 2x2 SVD through polar decomposition and a symmetric Givens eigen-solve.
// Returns U, V as (cos, sin) pairs of the rotation matrices
// U = [[cu, su], [-su, cu]] and V = [[cv, sv], [-sv, cv]] in row-major form,
// which is how svd2x2_modified hands Eigen the column-major Givens fill.
struct Svd64 { double cu, su, cv, sv, s0, s1; };

__device__ __forceinline__ Svd64 svd2x2_64(const M2d &A)
{
    // column-major view of A: {a00, a10, a01, a11}
    double c0 = A.a00, c1 = A.a10, c2 = A.a01, c3 = A.a11;
    double x0 = c0 + c3, x1 = c1 - c2;
    double den = sqrt(x0 * x0 + x1 * x1);
    double rc = 1.0, rs = 0.0;
    if (den != 0) {
        rc = x0 / den;
        rs = -x1 / den;
    }
    // s = G^T-rotated copy (rows 0,1 of each column)
    double s0 = rc * c0 - rs * c1;
    double s2 = rc * c2 - rs * c3;
    double s3 = rs * c2 + rc * c3;
    double x = s0, y = s2, z = s3;
    double y2 = y * y;
    double cosine, sine, sg0, sg1;
    if (y2 == 0) {
        cosine = 1;
        sine = 0;
        sg0 = x;
        sg1 = z;
    } else {
        double tau = 0.5 * (x - z);
        double w = sqrt(tau * tau + y2);
        double t = (tau > 0) ? y / (tau + w) : y / (tau - w);
        cosine = 1.0 / sqrt(t * t + 1.0);
        sine = -t * cosine;
        double cc = cosine * cosine;
        double csy = 2 * cosine * sine * y;
        double ss = sine * sine;
        sg0 = cc * x - csy + ss * z;
        sg1 = ss * x + csy + cc * z;
    }
    double vc, vs;
    if (sg0 < sg1) {
        double tmp = sg0;
        sg0 = sg1;
        sg1 = tmp;
        vc = -sine;
        vs = cosine;
    } else {
        vc = cosine;
        vs = sine;
    }
    double uc = rc * vc - rs * vs;
    double us = rs * vc + rc * vs;
    return {uc, us, vc, vs, sg0, sg1};
}

// U diag(s) V^T with U = [[cu, su], [-su, cu]], V = [[cv, sv], [-sv, cv]].
__device__ __forceinline__ M2d usvt64(const Svd64 &d, double t0, double t1)
{
    double U00 = d.cu, U01 = d.su, U10 = -d.su, U11 = d.cu;
    double V00 = d.cv, V01 = d.sv, V10 = -d.sv, V11 = d.cv;
    return {U00 * t0 * V00 + U01 * t1 * V01, U00 * t0 * V10 + U01 * t1 * V11,
            U10 * t0 * V00 + U11 * t1 * V01, U10 * t0 * V10 + U11 * t1 * V11};
}

struct Grain64 { double pmin, pmax, qmax, beta, mSq; };

// GetParametersForGrain (gpu_implementation5.cu:97-105) depends on the grain
// id only through these three C remainders (negative for negative ids).
struct GrainRes { int r21, r30, r11; };
__host__ __device__ __forceinline__ GrainRes grain_res(int grain) { return {grain % 21, (grain + 3) % 30, (grain + 4) % 11}; }

__device__ __forceinline__ Grain64 grain_params64(const icy_SimParams &P, GrainRes r)
{
    double var1 = 1.0 + P.GrainVariability * 0.05 * (-10 + r.r21);
    double var2 = 1.0 + P.GrainVariability * 0.033 * (-15 + r.r30);
    double var3 = 1.0 + P.GrainVariability * 0.1 * (-10 + r.r11);
    Grain64 g;
    g.pmax = P.IceCompressiveStrength * var1;
    g.pmin = -P.IceTensileStrength * var2;
    g.qmax = P.IceShearStrength * var3;
    g.beta = -g.pmin / g.pmax;
    g.mSq = (4 * g.qmax * g.qmax * (1 + 2 * g.beta)) / ((g.pmax * (1 + g.beta)) * (g.pmax * (1 + g.beta)));
    return g;
}

__device__ __forceinline__ bool outside_failure_surface64(const icy_SimParams &P, GrainRes grain, double p, double q)
{
    Grain64 g = grain_params64(P, grain);
    const double pmin2 = -3e6;
    if (p < 0) {
        if (p < pmin2) return true;
        double q0 = 2 * sqrt(-g.pmax * g.pmin) * g.qmax / (g.pmax - g.pmin);
        double k = -q0 / pmin2;
        double q_limit = k * (p - pmin2);
        return q > q_limit;
    }
    double yv = (1. + 2. * g.beta) * q * q + g.mSq * (p + g.beta * g.pmax) * (p - g.pmax);
    return yv > 0;
}

// Drucker-Prager projection of a crushed particle in principal space
// (Wolper_Drucker_Prager, gpu_implementation5.cu:48-94): from the trial
// singular values s0 >= s1 and Jp_inv, the new singular values and Jp_inv.
// changed = false when the state is left as it is (inside the yield surface).
struct DpResult { bool changed; double s0, s1, jp; };

__device__ __forceinline__ DpResult dp_project64(const icy_SimParams &P, double s0, double s1, double Jp_inv)
{
    const double mu = P.mu, kappa = P.kappa;
    const double Je_tr = s0 * s1;
    const double p_tr = -(kappa / 2.) * (Je_tr * Je_tr - 1.);
    const double sq0 = s0 * s0, sq1 = s1 * s1;
    const double half_sum = (sq0 + sq1) / 2;
    const double f = mu / Je_tr;
    const double sh0 = f * (sq0 - half_sum), sh1 = f * (sq1 - half_sum);
    const double q_tr = kCoeff1 * sqrt(sh0 * sh0 + sh1 * sh1);
    const double tan_phi = P.DP_tan_phi, p_thr = P.DP_threshold_p;
    const double pmax = P.IceCompressiveStrength, qmax = P.IceShearStrength;
    DpResult r{false, s0, s1, Jp_inv};
    if (p_tr < -p_thr || Jp_inv < 1) {
        double p_new = -p_thr;
        double Je_new = sqrt(-2. * p_new / kappa + 1.);
        double sn = sqrt(Je_new);
        r = {true, sn, sn, Jp_inv * (Je_new / Je_tr)};
    } else {
        double q_n_1;
        if (p_tr > pmax) {
            q_n_1 = 0;
        } else {
            double q_from_dp = (p_tr + p_thr) * tan_phi;
            q_n_1 = fmin(q_from_dp, qmax);
        }
        if (q_tr >= q_n_1) {
            double s_hat_n_1_norm = q_n_1 / kCoeff1;
            double n0 = sh0, n1 = sh1;
            double z = sh0 * sh0 + sh1 * sh1;
            if (z > 0) {
                double nn = sqrt(z);
                n0 /= nn;
                n1 /= nn;
            }
            double ff = s_hat_n_1_norm * (Je_tr / mu);
            double mean = (sq0 + sq1) / 2.0;
            r = {true, sqrt(ff * n0 + mean), sqrt(ff * n1 + mean), Jp_inv};
        }
    }
    return r;
}

// ComputePQ + failure check + Drucker-Prager map on the advected Fe.
// Updates Fe, Jp_inv and crushed in place; returns p_tr, q_tr.
__device__ __forceinline__ void constitutive64(const icy_SimParams &P, M2d &Fe, double &Jp_inv,
                                               uint8_t &crushed, GrainRes grain, double &p_tr, double &q_tr)
{
    const double mu = P.mu, kappa = P.kappa;
    Svd64 d = svd2x2_64(Fe);
    double Je_tr = d.s0 * d.s1;
    p_tr = -(kappa / 2.) * (Je_tr * Je_tr - 1.);
    double sq0 = d.s0 * d.s0, sq1 = d.s1 * d.s1;
    double half_sum = (sq0 + sq1) / 2;
    double f = mu / Je_tr;
    double sh0 = f * (sq0 - half_sum), sh1 = f * (sq1 - half_sum);
    q_tr = kCoeff1 * sqrt(sh0 * sh0 + sh1 * sh1);

    if (crushed == 0 && outside_failure_surface64(P, grain, p_tr, q_tr)) crushed = 1;
    if (crushed != 1) return;

    const DpResult r = dp_project64(P, d.s0, d.s1, Jp_inv);
    if (r.changed) {
        Fe = usvt64(d, r.s0, r.s1);
        Jp_inv = r.jp;
    }
}

// constitutive64 out of line, taking and returning values (a caller's hot
// loop keeps none of the SVD's registers and no state in local memory).
struct Cons64 { M2d F; double Jp, p, q; uint8_t crushed; };

static __device__ __noinline__ Cons64 constitutive64_call(const icy_SimParams &P, const M2d F, const double Jp,
                                                    const uint8_t crushed, const GrainRes grain)
{
    Cons64 o{F, Jp, 0.0, 0.0, crushed};
    constitutive64(P, o.F, o.Jp, o.crushed, grain, o.p, o.q);
    return o;
}

// The same update with ComputePQ's p and q of an intact particle taken from
// invariants of b = F F^T instead of the SVD: with J = det F and
// b - (tr b / 2) I = [[hd, b01], [b01, -hd]], the squared singular values
// differ by 2 |(hd, b01)|, so p = -kappa/2 (J^2 - 1) and
// q = sqrt(2) |mu/J dev(s^2)| = 2 (mu/J) sqrt(hd^2 + b01^2). An intact
// particle found inside its failure surface this way is done (Fe and
// Jp_inv unchanged); every other particle takes constitutive64 (SVD, the
// failure check again, the Drucker-Prager map). The results agree with
// constitutive64 to rounding (p, q within a few ulp); a particle within
// that rounding of its failure surface could be judged differently.
__device__ __forceinline__ void constitutive64_intact_first(const icy_SimParams &P, M2d &Fe, double &Jp_inv,
                                                            uint8_t &crushed, GrainRes grain, double &p_tr,
                                                            double &q_tr)
{
    if (crushed == 0) {
        const double Je = Fe.a00 * Fe.a11 - Fe.a10 * Fe.a01;
        const double b00 = Fe.a00 * Fe.a00 + Fe.a01 * Fe.a01, b11 = Fe.a10 * Fe.a10 + Fe.a11 * Fe.a11;
        const double b01 = Fe.a00 * Fe.a10 + Fe.a01 * Fe.a11, hd = 0.5 * (b00 - b11);
        const double p = -(P.kappa / 2.) * (Je * Je - 1.);
        const double q = 2.0 * (P.mu / Je) * sqrt(hd * hd + b01 * b01);
        if (Je > 0 && !outside_failure_surface64(P, grain, p, q)) {
            p_tr = p;
            q_tr = q;
            return;
        }
    }
    const Cons64 o = constitutive64_call(P, Fe, Jp_inv, crushed, grain);
    Fe = o.F;
    Jp_inv = o.Jp;
    crushed = o.crushed;
    p_tr = o.p;
    q_tr = o.q;
}

// Quadratic B-spline weights of v2_kernel_p2g / v2_kernel_g2p
// (gpu_implementation5.cu:185-193, 325-333): base node by truncation,
// fx in cell units relative to the base node.
struct Stencil64 { int bx, by; double fx, fy; double wx[3], wy[3]; };

__device__ __forceinline__ Stencil64 stencil64(double x, double y, double h_inv)
{
    Stencil64 s;
    s.bx = (int)(x * h_inv - 0.5);
    s.by = (int)(y * h_inv - 0.5);
    s.fx = x * h_inv - (double)s.bx;
    s.fy = y * h_inv - (double)s.by;
    double a0 = 1.5 - s.fx, a1 = s.fx - 1.0, a2 = s.fx - 0.5;
    s.wx[0] = 0.5 * a0 * a0;
    s.wx[1] = 0.75 - a1 * a1;
    s.wx[2] = 0.5 * a2 * a2;
    double b0 = 1.5 - s.fy, b1 = s.fy - 1.0, b2 = s.fy - 0.5;
    s.wy[0] = 0.5 * b0 * b0;
    s.wy[1] = 0.75 - b1 * b1;
    s.wy[2] = 0.5 * b2 * b2;
    return s;
}

// Grid-node velocity update of v2_kernel_update_nodes
// (gpu_implementation5.cu:221-289) for a node with mass > 0. Returns the
// reaction force on the indenter in f0/f1 and the angular bin (or -1).
struct NodeOut { double v0, v1, f0, f1; int bin; };

__device__ __forceinline__ NodeOut update_node64(const icy_SimParams &P, int ix, int iy, double mass,
                                                 double p0, double p1, double ind_x, double ind_y)
{
    const double dt = P.InitialTimeStep, cellsize = P.cellsize;
    NodeOut o;
    o.f0 = 0;
    o.f1 = 0;
    o.bin = -1;
    double v0 = p0 / mass, v1 = p1 / mass;
    v1 -= dt * P.Gravity;
    double vmax = 0.5 * cellsize / dt;
    double nrm = sqrt(v0 * v0 + v1 * v1);
    if (nrm > vmax) {
        v0 = v0 / nrm * vmax;
        v1 = v1 / nrm * vmax;
    }
    double n0 = ix * cellsize - ind_x;
    double n1 = iy * cellsize - ind_y;
    if (n0 * n0 + n1 * n1 < P.IndRSq) {
        const double vco0 = P.IndVelocity, vco1 = 0;
        double vr0 = v0 - vco0, vr1 = v1 - vco1;
        double z = n0 * n0 + n1 * n1;
        if (z > 0) {
            double nn = sqrt(z);
            n0 /= nn;
            n1 /= nn;
        }
        double vn = vr0 * n0 + vr1 * n1;
        if (vn < 0) {
            double vt0 = vr0 - n0 * vn, vt1 = vr1 - n1 * vn;
            double pv0 = v0, pv1 = v1;
            v0 = vco0 + vt0;
            v1 = vco1 + vt1;
            o.f0 = (pv0 - v0) * mass / dt;
            o.f1 = (pv1 - v1) * mass / dt;
            double angle = atan2(n0, n1);
            angle += ICM_PI;
            angle *= P.n_indenter_subdivisions / (2 * ICM_PI);
            int index = (int)angle;
            index = max(index, 0);
            index = min(index, P.n_indenter_subdivisions - 1);
            o.bin = index;
        }
    }
    if (iy <= 2) {
        v0 = 0;
        v1 = 0;
    } else if (iy >= P.GridY - 3 && v1 > 0) {
        v1 = 0;
    }
    if (ix <= 2 && v0 < 0)
        v0 = 0;
    else if (ix >= P.GridX - 3 && v0 > 0)
        v0 = 0;
    o.v0 = v0;
    o.v1 = v1;
    return o;
}

}  // namespace icm
