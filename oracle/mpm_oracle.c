/*
 * mpm_oracle.c -- CPU FP64 restatement of iceMPM's 2D MLS-MPM substep.
 *
 * TEST INFRASTRUCTURE. This file is the checker for the CUDA kernels in
 * icempm_b200/csrc and the timed CPU baseline of bench.py. Only tests/,
 * __graft_entry__.smoke() and bench.py (its CPU-baseline and reference legs)
 * may load it. The product never calls it.
 *
 * What it restates (paths inside the iceMPM project):
 *   simulation/gpu_implementation5.cu:21-22   coeff1 = sqrt(2)
 *   simulation/gpu_implementation5.cu:24-34   KirchhoffStress_Wolper
 *   simulation/gpu_implementation5.cu:36-44   ComputePQ
 *   simulation/gpu_implementation5.cu:48-94   Wolper_Drucker_Prager
 *   simulation/gpu_implementation5.cu:97-111  GetParametersForGrain
 *   simulation/gpu_implementation5.cu:114-141 CheckIfPointIsInsideFailureSurface
 *   simulation/gpu_implementation5.cu:148-213 v2_kernel_p2g
 *   simulation/gpu_implementation5.cu:215-290 v2_kernel_update_nodes
 *   simulation/gpu_implementation5.cu:294-379 v2_kernel_g2p
 *   simulation/gpu_implementation5.cu:386-416 dev_d, dev, svd, svd2x2_modified
 *   simulation/helper_math.cuh:27-46,81-140   polar_decomposition, singular_value_decomposition
 *   simulation/givens.cuh:100-128,161-166     GivensRotation fill / mat_rotation / operator*=
 *   simulation/model.cpp:11-47                Model::Step substep loop
 *
 * Eigen behaviour the device code relies on and that is reproduced here:
 *   normalize()/normalized() leave a zero vector unchanged; cast<int>()
 *   truncates toward zero; determinant = a00*a11 - a10*a01; products are
 *   evaluated left to right as written.
 *
 * Deliberate deviation: the reference adds P2G contributions of a stencil
 * node that lies outside the grid at an out-of-range index (undefined
 * behaviour) after raising gpu_error_indicator (gpu_implementation5.cu:206).
 * Here such contributions are dropped and the error indicator is raised; G2P
 * reads an out-of-grid node as zero velocity.
 *
 * Parity pin: every function above and the whole substep are checked
 * against the reference's own code compiled for the host
 * (oracle/build_ref.sh: helper_math.cuh/givens.cuh into libref_svd.so;
 * gpu_implementation5.cu:1-416 with an Eigen-subset stub into
 * libref_step.so). With one thread the results agree bit for bit on scenes
 * whose stencils stay inside the grid; the force bins, which this file sums
 * per substep before adding them, agree to rounding.
 *
 * Parallelism: OpenMP. P2G scatters into per-thread private node bands that
 * are summed in thread order, so results are deterministic for a fixed
 * thread count; with one thread the summation order is particle order.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "../include/icempm_params.h"

#define COEFF1 1.4142135623730950 /* sqrt((6-d)/2) with d = 2 */

/* ---------------------------------------------------------------- SVD 2x2 */

typedef struct { double c, s; } givens_t; /* rotation rows (0,1) */

/* Column-major 2x2 "row rotation" G^T A of givens.cuh:120-128. */
static void givens_mat_rotation(givens_t g, double a[4])
{
    for (int d = 0; d < 2; d++) {
        double tau1 = a[0 + d * 2];
        double tau2 = a[1 + d * 2];
        a[0 + d * 2] = g.c * tau1 - g.s * tau2;
        a[1 + d * 2] = g.s * tau1 + g.c * tau2;
    }
}

/* givens.cuh:161-166 */
static void givens_mul(givens_t *self, givens_t a)
{
    double new_c = self->c * a.c - self->s * a.s;
    double new_s = self->s * a.c + self->c * a.s;
    self->c = new_c;
    self->s = new_s;
}

/* givens.cuh:100-111 for Dim = 2: column-major {c, s, -s, c}. */
static void givens_fill(givens_t g, double a[4])
{
    a[0] = g.c;
    a[1] = g.s;
    a[2] = -g.s;
    a[3] = g.c;
}

/* helper_math.cuh:27-46 */
static void polar_decomposition(const double a[4], givens_t *r, double s[4])
{
    double x0 = a[0] + a[3];
    double x1 = a[1] - a[2];
    double denominator = sqrt(x0 * x0 + x1 * x1);
    r->c = 1.0;
    r->s = 0.0;
    if (denominator != 0) {
        r->c = x0 / denominator;
        r->s = -x1 / denominator;
    }
    for (int i = 0; i < 4; ++i) s[i] = a[i];
    givens_mat_rotation(*r, s);
}

/* helper_math.cuh:81-140 (input aa in the order svd2x2_modified passes it) */
static void singular_value_decomposition(const double aa[4], givens_t *u,
                                         double sigma[2], givens_t *v)
{
    double s_sym[4];
    double a[4] = {aa[0], aa[2], aa[1], aa[3]};
    polar_decomposition(a, u, s_sym);
    double cosine, sine;
    double x = s_sym[0];
    double y = s_sym[2];
    double z = s_sym[3];
    double y2 = y * y;
    if (y2 == 0) {
        cosine = 1;
        sine = 0;
        sigma[0] = x;
        sigma[1] = z;
    } else {
        double tau = 0.5 * (x - z);
        double w = sqrt(tau * tau + y2);
        double t;
        if (tau > 0)
            t = y / (tau + w);
        else
            t = y / (tau - w);
        cosine = 1.0 / sqrt(t * t + 1.0);
        sine = -t * cosine;
        double c2 = cosine * cosine;
        double csy = 2 * cosine * sine * y;
        double s2 = sine * sine;
        sigma[0] = c2 * x - csy + s2 * z;
        sigma[1] = s2 * x + csy + c2 * z;
    }
    if (sigma[0] < sigma[1]) {
        double tmp = sigma[0];
        sigma[0] = sigma[1];
        sigma[1] = tmp;
        v->c = -sine;
        v->s = cosine;
    } else {
        v->c = cosine;
        v->s = sine;
    }
    givens_mul(u, *v);
}

/* gpu_implementation5.cu:399-416. A, U, V row-major 2x2 (Eigen's comma
 * initializer fills row by row). */
void oracle_svd2x2(const double A[4], double U[4], double S[2], double V[4])
{
    givens_t gu = {1.0, 0.0}, gv = {1.0, 0.0};
    double a[4] = {A[0], A[1], A[2], A[3]};
    double u[4], v[4];
    singular_value_decomposition(a, &gu, S, &gv);
    givens_fill(gu, u);
    givens_fill(gv, v);
    for (int i = 0; i < 4; i++) {
        U[i] = u[i];
        V[i] = v[i];
    }
}

/* ----------------------------------------------------- constitutive model */

/* gpu_implementation5.cu:24-34 and dev() at :391-394. F, tau row-major. */
void oracle_kirchhoff(const icy_SimParams *P, const double F[4], double tau[4])
{
    const double kappa = P->kappa, mu = P->mu;
    double Je = F[0] * F[3] - F[2] * F[1];
    double b00 = F[0] * F[0] + F[1] * F[1];
    double b01 = F[0] * F[2] + F[1] * F[3];
    double b10 = F[2] * F[0] + F[3] * F[1];
    double b11 = F[2] * F[2] + F[3] * F[3];
    double half_tr = (b00 + b11) / 2;
    double s1 = mu * (1 / Je);
    double s2 = kappa * (Je * Je - 1.);
    tau[0] = s1 * (b00 - half_tr) + s2;
    tau[1] = s1 * b01;
    tau[2] = s1 * b10;
    tau[3] = s1 * (b11 - half_tr) + s2;
}

typedef struct {
    double U[4], V[4], S[2], S2[2], s_hat[2];
    double Je_tr, p_tr, q_tr;
} pq_t;

/* gpu_implementation5.cu:36-44 and dev_d() at :386-389 */
static void compute_pq(const icy_SimParams *P, const double Fe[4], pq_t *o)
{
    oracle_svd2x2(Fe, o->U, o->S, o->V);
    o->Je_tr = o->S[0] * o->S[1];
    o->p_tr = -(P->kappa / 2.) * (o->Je_tr * o->Je_tr - 1.);
    o->S2[0] = o->S[0] * o->S[0];
    o->S2[1] = o->S[1] * o->S[1];
    double half_sum = (o->S2[0] + o->S2[1]) / 2;
    double f = P->mu / o->Je_tr;
    o->s_hat[0] = f * (o->S2[0] - half_sum);
    o->s_hat[1] = f * (o->S2[1] - half_sum);
    o->q_tr = COEFF1 * sqrt(o->s_hat[0] * o->s_hat[0] + o->s_hat[1] * o->s_hat[1]);
}

/* gpu_implementation5.cu:97-111 */
static void grain_params(const icy_SimParams *P, short grain, double *pmin,
                         double *pmax, double *qmax, double *beta, double *mSq)
{
    double var1 = 1.0 + P->GrainVariability * 0.05 * (-10 + grain % 21);
    double var2 = 1.0 + P->GrainVariability * 0.033 * (-15 + (grain + 3) % 30);
    double var3 = 1.0 + P->GrainVariability * 0.1 * (-10 + (grain + 4) % 11);
    *pmax = P->IceCompressiveStrength * var1;
    *pmin = -P->IceTensileStrength * var2;
    *qmax = P->IceShearStrength * var3;
    *beta = -*pmin / *pmax;
    *mSq = (4 * *qmax * *qmax * (1 + 2 * *beta)) /
           ((*pmax * (1 + *beta)) * (*pmax * (1 + *beta)));
}

/* gpu_implementation5.cu:114-141; returns the new crushed flag. */
static int failure_check(const icy_SimParams *P, short grain, double p, double q)
{
    double beta, M_sq, pmin, pmax, qmax;
    grain_params(P, grain, &pmin, &pmax, &qmax, &beta, &M_sq);
    const double pmin2 = -3e6;
    if (p < 0) {
        if (p < pmin2) return 1;
        double q0 = 2 * sqrt(-pmax * pmin) * qmax / (pmax - pmin);
        double k = -q0 / pmin2;
        double q_limit = k * (p - pmin2);
        if (q > q_limit) return 1;
    } else {
        double y = (1. + 2. * beta) * q * q + M_sq * (p + beta * pmax) * (p - pmax);
        if (y > 0) return 1;
    }
    return 0;
}

/* U diag(s) V^T, row-major */
static void usvt(const double U[4], const double s[2], const double V[4], double F[4])
{
    for (int k = 0; k < 2; k++)
        for (int m = 0; m < 2; m++)
            F[k * 2 + m] = U[k * 2 + 0] * s[0] * V[m * 2 + 0] + U[k * 2 + 1] * s[1] * V[m * 2 + 1];
}

/* gpu_implementation5.cu:48-94 */
static void drucker_prager(const icy_SimParams *P, const pq_t *o, double Fe[4], double *Jp_inv)
{
    const double mu = P->mu, kappa = P->kappa;
    const double tan_phi = P->DP_tan_phi, p_thr = P->DP_threshold_p;
    const double pmax = P->IceCompressiveStrength, qmax = P->IceShearStrength;
    if (o->p_tr < -p_thr || *Jp_inv < 1) {
        double p_new = -p_thr;
        double Je_new = sqrt(-2. * p_new / kappa + 1.);
        double sn = sqrt(Je_new);
        double s_new[2] = {sn, sn};
        usvt(o->U, s_new, o->V, Fe);
        *Jp_inv *= Je_new / o->Je_tr;
    } else {
        double q_n_1;
        if (o->p_tr > pmax) {
            q_n_1 = 0;
        } else {
            double q_from_dp = (o->p_tr + p_thr) * tan_phi;
            q_n_1 = q_from_dp < qmax ? q_from_dp : qmax;
        }
        if (o->q_tr >= q_n_1) {
            double s_hat_n_1_norm = q_n_1 / COEFF1;
            double nrm2 = o->s_hat[0] * o->s_hat[0] + o->s_hat[1] * o->s_hat[1];
            double n0 = o->s_hat[0], n1 = o->s_hat[1];
            if (nrm2 > 0) {
                double nrm = sqrt(nrm2);
                n0 /= nrm;
                n1 /= nrm;
            }
            double f = s_hat_n_1_norm * (o->Je_tr / mu);
            double mean = (o->S2[0] + o->S2[1]) / 2.0;
            double s_new[2] = {sqrt(f * n0 + mean), sqrt(f * n1 + mean)};
            usvt(o->U, s_new, o->V, Fe);
        }
    }
}

/* Exports of the single functions for the per-function pin against the
 * reference's own code (tests/test_oracle.py). out: U[4], sigma[2], V[4],
 * Je_tr, p_tr, q_tr, sigma^2[2], s_hat[2] (17 doubles). */
void oracle_compute_pq(const icy_SimParams *P, const double Fe[4], double out[17])
{
    pq_t o;
    compute_pq(P, Fe, &o);
    for (int i = 0; i < 4; i++) {
        out[i] = o.U[i];
        out[6 + i] = o.V[i];
    }
    out[4] = o.S[0];
    out[5] = o.S[1];
    out[10] = o.Je_tr;
    out[11] = o.p_tr;
    out[12] = o.q_tr;
    out[13] = o.S2[0];
    out[14] = o.S2[1];
    out[15] = o.s_hat[0];
    out[16] = o.s_hat[1];
}

/* out: pmin, pmax, qmax, beta, mSq */
void oracle_grain_params(const icy_SimParams *P, short grain, double out[5])
{
    grain_params(P, grain, &out[0], &out[1], &out[2], &out[3], &out[4]);
}

int oracle_failure_check(const icy_SimParams *P, short grain, double p, double q)
{
    return failure_check(P, grain, p, q);
}

/* The part of v2_kernel_g2p after the Fe update (gpu_implementation5.cu:353-356):
 * ComputePQ, failure check for intact points, DP map for crushed points. */
void oracle_constitutive(const icy_SimParams *P, double Fe[4], double *Jp_inv,
                         uint8_t *crushed, short grain, double *p_tr, double *q_tr)
{
    pq_t o;
    compute_pq(P, Fe, &o);
    if (*crushed == 0 && failure_check(P, grain, o.p_tr, o.q_tr)) *crushed = 1;
    if (*crushed == 1) drucker_prager(P, &o, Fe, Jp_inv);
    *p_tr = o.p_tr;
    *q_tr = o.q_tr;
}

/* ------------------------------------------------------------- kernels */

#define ROW(pts, P, r) ((pts) + (size_t)(r) * (P)->nPtsPitch)

static inline uint8_t get_crushed(const double *pts, int i) { return ((const uint8_t *)pts)[i]; }
static inline short get_grain(const icy_SimParams *P, const double *pts, int i)
{
    const short *g = (const short *)((const char *)pts + P->nPtsPitch);
    return g[i];
}

/* cuda_reset_grid (gpu_implementation5.cu:554-559) */
void oracle_reset_grid(const icy_SimParams *P, double *grid)
{
    memset(grid, 0, sizeof(double) * P->nGridPitch * ICM_N_GRID_ARRAYS);
}

/* One particle's P2G scatter (gpu_implementation5.cu:165-212) into a node
 * window [lo, lo+len) of 3 rows with row stride `stride`. Returns 1 if a
 * stencil node lies outside the grid. */
static int p2g_particle(const icy_SimParams *P, const double *pts, int pt,
                        double *win, long lo, long len, size_t stride)
{
    const double dt = P->InitialTimeStep, vol = P->ParticleVolume, h = P->cellsize;
    const double h_inv = P->cellsize_inv, Dinv = P->Dp_inv, m = P->ParticleMass;
    const int gridX = P->GridX, gridY = P->GridY;
    double pos[2], vel[2], Fe[4], Bp[4];
    for (int i = 0; i < 2; i++) {
        pos[i] = ROW(pts, P, ICM_IDX_POSX + i)[pt];
        vel[i] = ROW(pts, P, ICM_IDX_VELX + i)[pt];
        for (int j = 0; j < 2; j++) {
            Fe[i * 2 + j] = ROW(pts, P, ICM_IDX_FE00 + i * 2 + j)[pt];
            Bp[i * 2 + j] = ROW(pts, P, ICM_IDX_BP00 + i * 2 + j)[pt];
        }
    }
    double tau[4];
    oracle_kirchhoff(P, Fe, tau);
    double c = (dt * vol) * Dinv;
    double st[4];
    for (int k = 0; k < 4; k++) st[k] = m * Bp[k] - c * tau[k];

    int base[2];
    double fx[2], ww[3][2];
    for (int k = 0; k < 2; k++) {
        base[k] = (int)(pos[k] * h_inv - 0.5);
        fx[k] = pos[k] * h_inv - (double)base[k];
        double v0 = 1.5 - fx[k], v1 = fx[k] - 1.0, v2 = fx[k] - 0.5;
        ww[0][k] = 0.5 * v0 * v0;
        ww[1][k] = 0.75 - v1 * v1;
        ww[2][k] = 0.5 * v2 * v2;
    }
    int err = 0;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double Wip = ww[i][0] * ww[j][1];
            double d0 = (i - fx[0]) * h, d1 = (j - fx[1]) * h;
            double incV0 = Wip * (vel[0] * m + (st[0] * d0 + st[1] * d1));
            double incV1 = Wip * (vel[1] * m + (st[2] * d0 + st[3] * d1));
            double incM = Wip * m;
            int i2 = i + base[0], j2 = j + base[1];
            if (i2 < 0 || j2 < 0 || i2 >= gridX || j2 >= gridY) {
                err = 1;
                continue;
            }
            long idx = (long)i2 + (long)j2 * gridX - lo;
            if (idx < 0 || idx >= len) continue; /* cannot happen: window covers the stencil */
            win[idx] += incM;
            win[stride + idx] += incV0;
            win[2 * stride + idx] += incV1;
        }
    return err;
}

static void stencil_range(const icy_SimParams *P, const double *pts, int pt, long *lo, long *hi)
{
    const double h_inv = P->cellsize_inv;
    int b0 = (int)(ROW(pts, P, ICM_IDX_POSX)[pt] * h_inv - 0.5);
    int b1 = (int)(ROW(pts, P, ICM_IDX_POSX + 1)[pt] * h_inv - 0.5);
    long a = (long)b0 + (long)b1 * P->GridX;
    long b = (long)(b0 + 2) + (long)(b1 + 2) * P->GridX;
    if (a < 0) a = 0;
    if (b > (long)P->GridTotal - 1) b = (long)P->GridTotal - 1;
    *lo = a;
    *hi = b;
}

/* v2_kernel_p2g over all particles. grid: 3 rows x nGridPitch. Returns the
 * error indicator (1 if any stencil node left the grid). */
int oracle_p2g(const icy_SimParams *P, const double *pts, double *grid, int nthreads)
{
    const int n = P->nPts;
    const size_t gp = P->nGridPitch;
    if (nthreads <= 1 || n < 4096) {
        int err = 0;
        for (int pt = 0; pt < n; pt++) err |= p2g_particle(P, pts, pt, grid, 0, (long)gp, gp);
        return err;
    }
    int T = nthreads;
    long *lo = (long *)calloc(T, sizeof(long));
    long *hi = (long *)calloc(T, sizeof(long));
    double **win = (double **)calloc(T, sizeof(double *));
    int err = 0;
#pragma omp parallel num_threads(T) reduction(| : err)
    {
#ifdef _OPENMP
        int t = omp_get_thread_num();
#else
        int t = 0;
#endif
        int p0 = (int)((long)n * t / T), p1 = (int)((long)n * (t + 1) / T);
        long l = (long)P->GridTotal, hgh = -1;
        for (int pt = p0; pt < p1; pt++) {
            long a, b;
            stencil_range(P, pts, pt, &a, &b);
            if (a < l) l = a;
            if (b > hgh) hgh = b;
        }
        if (hgh < l) { l = 0; hgh = -1; }
        long len = hgh - l + 1;
        lo[t] = l;
        hi[t] = hgh;
        win[t] = len > 0 ? (double *)calloc((size_t)len * 3, sizeof(double)) : NULL;
        for (int pt = p0; pt < p1; pt++) err |= p2g_particle(P, pts, pt, win[t], l, len, (size_t)len);
#pragma omp barrier
#pragma omp for schedule(static)
        for (long node = 0; node < (long)P->GridTotal; node++) {
            for (int s = 0; s < T; s++) {
                if (node < lo[s] || node > hi[s]) continue;
                long len_s = hi[s] - lo[s] + 1;
                long k = node - lo[s];
                grid[node] += win[s][k];
                grid[gp + node] += win[s][len_s + k];
                grid[2 * gp + node] += win[s][2 * len_s + k];
            }
        }
    }
    for (int t = 0; t < T; t++) free(win[t]);
    free(win);
    free(lo);
    free(hi);
    return err;
}

/* One node of v2_kernel_update_nodes (gpu_implementation5.cu:215-290).
 * Adds its indenter reaction to bins (2*nsub) and to total[2]. */
static void update_node(const icy_SimParams *P, double *grid, long idx, double ix,
                        double iy, double *bins, double *total)
{
    double mass = grid[idx];
    if (mass == 0) return;
    const size_t gp = P->nGridPitch;
    const double gravity = P->Gravity, indRsq = P->IndRSq, dt = P->InitialTimeStep;
    const double ind_velocity = P->IndVelocity, cellsize = P->cellsize;
    const int gridX = P->GridX, gridY = P->GridY;
    const double vco0 = ind_velocity, vco1 = 0;
    double v0 = grid[gp + idx], v1 = grid[2 * gp + idx];
    v0 /= mass;
    v1 /= mass;
    v1 -= dt * gravity;
    double vmax = 0.5 * cellsize / dt;
    double vn2 = sqrt(v0 * v0 + v1 * v1);
    if (vn2 > vmax) {
        double nv = sqrt(v0 * v0 + v1 * v1);
        v0 = v0 / nv * vmax;
        v1 = v1 / nv * vmax;
    }
    int idx_x = (int)(idx % gridX);
    int idx_y = (int)(idx / gridX);
    double n0 = idx_x * cellsize - ix;
    double n1 = idx_y * cellsize - iy;
    if (n0 * n0 + n1 * n1 < indRsq) {
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
            double f0 = (pv0 - v0) * mass / dt;
            double f1 = (pv1 - v1) * mass / dt;
            double angle = atan2(n0, n1);
            angle += ICM_PI;
            angle *= P->n_indenter_subdivisions / (2 * ICM_PI);
            int index = (int)angle;
            if (index < 0) index = 0;
            if (index > P->n_indenter_subdivisions - 1) index = P->n_indenter_subdivisions - 1;
            bins[2 * index] += f0;
            bins[2 * index + 1] += f1;
            total[0] += f0;
            total[1] += f1;
        }
    }
    if (idx_y <= 2) {
        v0 = 0;
        v1 = 0;
    } else if (idx_y >= gridY - 3 && v1 > 0)
        v1 = 0;
    if (idx_x <= 2 && v0 < 0)
        v0 = 0;
    else if (idx_x >= gridX - 3 && v0 > 0)
        v0 = 0;
    grid[gp + idx] = v0;
    grid[2 * gp + idx] = v1;
}

/* v2_kernel_update_nodes over all nodes. bins: 2*n_indenter_subdivisions;
 * total (may be NULL): this substep's summed reaction force. */
void oracle_update_nodes(const icy_SimParams *P, double *grid, double *bins, double ix,
                         double iy, double *total, int nthreads)
{
    const int nsub2 = 2 * P->n_indenter_subdivisions;
    double tot[2] = {0, 0};
    int T = nthreads < 1 ? 1 : nthreads;
    double *tb = (double *)calloc((size_t)T * (nsub2 + 2), sizeof(double));
#pragma omp parallel num_threads(T)
    {
#ifdef _OPENMP
        int t = omp_get_thread_num();
#else
        int t = 0;
#endif
        double *mb = tb + (size_t)t * (nsub2 + 2);
        long n = P->GridTotal;
        long a = n * t / T, b = n * (t + 1) / T;
        for (long idx = a; idx < b; idx++) update_node(P, grid, idx, ix, iy, mb, mb + nsub2);
    }
    for (int t = 0; t < T; t++) {
        double *mb = tb + (size_t)t * (nsub2 + 2);
        for (int k = 0; k < nsub2; k++) bins[k] += mb[k];
        tot[0] += mb[nsub2];
        tot[1] += mb[nsub2 + 1];
    }
    free(tb);
    if (total) {
        total[0] = tot[0];
        total[1] = tot[1];
    }
}

/* One particle of v2_kernel_g2p (gpu_implementation5.cu:294-379). */
static void g2p_particle(const icy_SimParams *P, double *pts, const double *grid, int pt, int recordPQ)
{
    const size_t gp = P->nGridPitch;
    const double h_inv = P->cellsize_inv, dt = P->InitialTimeStep;
    const int gridX = P->GridX, gridY = P->GridY;
    double pos[2], Fe[4], vel[2] = {0, 0}, Bp[4] = {0, 0, 0, 0};
    for (int i = 0; i < 2; i++) {
        pos[i] = ROW(pts, P, ICM_IDX_POSX + i)[pt];
        for (int j = 0; j < 2; j++) Fe[i * 2 + j] = ROW(pts, P, ICM_IDX_FE00 + i * 2 + j)[pt];
    }
    uint8_t crushed = get_crushed(pts, pt);
    short grain = get_grain(P, pts, pt);
    double Jp_inv = ROW(pts, P, ICM_IDX_JP_INV)[pt];

    int base[2];
    double fx[2], ww[3][2];
    for (int k = 0; k < 2; k++) {
        base[k] = (int)(pos[k] * h_inv - 0.5);
        fx[k] = pos[k] * h_inv - (double)base[k];
        double v0 = 1.5 - fx[k], v1 = fx[k] - 1.0, v2 = fx[k] - 0.5;
        ww[0][k] = 0.5 * v0 * v0;
        ww[1][k] = 0.75 - v1 * v1;
        ww[2][k] = 0.5 * v2 * v2;
    }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            double d0 = i - fx[0], d1 = j - fx[1];
            double weight = ww[i][0] * ww[j][1];
            int i2 = i + base[0], j2 = j + base[1];
            double nv0 = 0, nv1 = 0;
            if (i2 >= 0 && j2 >= 0 && i2 < gridX && j2 < gridY) {
                long idx = (long)i2 + (long)j2 * gridX;
                nv0 = grid[gp + idx];
                nv1 = grid[2 * gp + idx];
            }
            vel[0] += weight * nv0;
            vel[1] += weight * nv1;
            double c = (4. * h_inv) * weight;
            Bp[0] += c * (nv0 * d0);
            Bp[1] += c * (nv0 * d1);
            Bp[2] += c * (nv1 * d0);
            Bp[3] += c * (nv1 * d1);
        }
    pos[0] += vel[0] * dt;
    pos[1] += vel[1] * dt;
    double M[4] = {1 + dt * Bp[0], dt * Bp[1], dt * Bp[2], 1 + dt * Bp[3]};
    double Fn[4];
    for (int k = 0; k < 2; k++)
        for (int m = 0; m < 2; m++) Fn[k * 2 + m] = M[k * 2 + 0] * Fe[0 * 2 + m] + M[k * 2 + 1] * Fe[1 * 2 + m];

    double p_tr, q_tr;
    oracle_constitutive(P, Fn, &Jp_inv, &crushed, grain, &p_tr, &q_tr);

    ROW(pts, P, ICM_IDX_JP_INV)[pt] = Jp_inv;
    for (int i = 0; i < 2; i++) {
        ROW(pts, P, ICM_IDX_POSX + i)[pt] = pos[i];
        ROW(pts, P, ICM_IDX_VELX + i)[pt] = vel[i];
        for (int j = 0; j < 2; j++) {
            ROW(pts, P, ICM_IDX_FE00 + i * 2 + j)[pt] = Fn[i * 2 + j];
            ROW(pts, P, ICM_IDX_BP00 + i * 2 + j)[pt] = Bp[i * 2 + j];
        }
    }
    ((uint8_t *)pts)[pt] = crushed;
    if (recordPQ) {
        ROW(pts, P, ICM_IDX_P)[pt] = p_tr;
        ROW(pts, P, ICM_IDX_Q)[pt] = q_tr;
    }
}

void oracle_g2p(const icy_SimParams *P, double *pts, const double *grid, int recordPQ, int nthreads)
{
    int T = nthreads < 1 ? 1 : nthreads;
#pragma omp parallel for num_threads(T) schedule(static)
    for (int pt = 0; pt < P->nPts; pt++) g2p_particle(P, pts, grid, pt, recordPQ);
}

/* Runs n substeps of Model::Step's loop (model.cpp:20-29) starting from
 * P->SimulationStep / P->SimulationTime and advances both. Force bins are
 * accumulated (the caller resets them per frame, model.cpp:18);
 * force_hist (may be NULL) receives 2 doubles per substep: that substep's
 * summed indenter reaction. Returns the OR of the P2G error indicators. */
int oracle_run_substeps(icy_SimParams *P, double *pts, double *grid, double *bins,
                        double *force_hist, int n, int nthreads)
{
    double t = P->SimulationTime;
    int err = 0;
    for (int k = 1; k <= n; k++) {
        t += P->InitialTimeStep;
        P->indenter_x = P->indenter_x_initial + t * P->IndVelocity;
        oracle_reset_grid(P, grid);
        err |= oracle_p2g(P, pts, grid, nthreads);
        double tot[2];
        oracle_update_nodes(P, grid, bins, P->indenter_x, P->indenter_y, tot, nthreads);
        if (force_hist) {
            force_hist[2 * (k - 1)] = tot[0];
            force_hist[2 * (k - 1) + 1] = tot[1];
        }
        oracle_g2p(P, pts, grid, (P->SimulationStep + k) % P->UpdateEveryNthStep == 0, nthreads);
    }
    P->SimulationStep += n;
    P->SimulationTime = t;
    return err;
}

int oracle_max_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
