/*
 * scene_oracle.c -- the seeded synthetic ice block of the benchmark
 * workloads, restated for the CPU arm of bench.py so that the arm builds its
 * input without the product library.
 *
 * TEST INFRASTRUCTURE, like mpm_oracle.c: only tests/ and bench.py's CPU legs
 * load it. It follows the product's icm_scene_block
 * (icempm_b200/csrc/scene.cpp), which stands in for
 * SnapshotManager::LoadRawPoints (simulation/snapshotmanager.cpp:186-286):
 *   - a jittered lattice of 2x2 sites per cell, each site moved by up to a
 *     quarter of the site spacing, drawn from std::mt19937_64 (the 64-bit
 *     Mersenne Twister of Matsumoto and Nishimura, restated below) as
 *     (g() >> 11) * 2^-53;
 *   - Voronoi grains from seeds drawn from the same stream, found by a ring
 *     search over a bucket grid (ties to the lower seed);
 *   - the LoadRawPoints pipeline: float32 points, a stable sort by the
 *     SortPoints key (snapshotmanager.cpp:288-304), bounding box and block
 *     coordinates (:229-240, parameters_sim.cpp:149-155), the block centred
 *     in x and lifted by 2h (:244-250), offsets added in float (:275-276),
 *     Volume / ParticleVolume / ParticleMass (:225-242, 267-268);
 *   - the indenter just touching the block's left face at a given height
 *     (the synthetic block's documented placement).
 * A CPU test holds the result bit-identical to icm_scene_block.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../include/icempm_params.h"

/* ------------------------------------------------ 64-bit Mersenne Twister */

#define MT_N 312
#define MT_M 156

typedef struct {
    uint64_t mt[MT_N];
    int i;
} mt64_t;

static void mt64_seed(mt64_t *g, uint64_t seed)
{
    g->mt[0] = seed;
    for (int i = 1; i < MT_N; i++)
        g->mt[i] = 6364136223846793005ULL * (g->mt[i - 1] ^ (g->mt[i - 1] >> 62)) + (uint64_t)i;
    g->i = MT_N;
}

static uint64_t mt64_next(mt64_t *g)
{
    static const uint64_t mag[2] = {0ULL, 0xB5026F5AA96619E9ULL};
    const uint64_t UM = 0xFFFFFFFF80000000ULL, LM = 0x7FFFFFFFULL;
    if (g->i >= MT_N) {
        int k;
        uint64_t x;
        for (k = 0; k < MT_N - MT_M; k++) {
            x = (g->mt[k] & UM) | (g->mt[k + 1] & LM);
            g->mt[k] = g->mt[k + MT_M] ^ (x >> 1) ^ mag[x & 1ULL];
        }
        for (; k < MT_N - 1; k++) {
            x = (g->mt[k] & UM) | (g->mt[k + 1] & LM);
            g->mt[k] = g->mt[k + (MT_M - MT_N)] ^ (x >> 1) ^ mag[x & 1ULL];
        }
        x = (g->mt[MT_N - 1] & UM) | (g->mt[0] & LM);
        g->mt[MT_N - 1] = g->mt[MT_M - 1] ^ (x >> 1) ^ mag[x & 1ULL];
        g->i = 0;
    }
    uint64_t x = g->mt[g->i++];
    x ^= (x >> 29) & 0x5555555555555555ULL;
    x ^= (x << 17) & 0x71D67FFFEDA60000ULL;
    x ^= (x << 37) & 0xFFF7EEE000000000ULL;
    x ^= (x >> 43);
    return x;
}

static double u01(mt64_t *g) { return (double)(mt64_next(g) >> 11) * (1.0 / 9007199254740992.0); }

/* ------------------------------------------------------------- the block */

typedef struct {
    float x, y;
    short g;
    int order; /* input position: ties of the sort keep it */
    int key;
} raw_point_t;

static int cmp_key(const void *a, const void *b)
{
    const raw_point_t *p = (const raw_point_t *)a, *q = (const raw_point_t *)b;
    if (p->key != q->key) return p->key < q->key ? -1 : 1;
    return p->order < q->order ? -1 : (p->order > q->order);
}

static int imax(int a, int b) { return a > b ? a : b; }
static int imin(int a, int b) { return a < b ? a : b; }

/* The block of cells_x x cells_y cells at 4 points per cell. P must hold the
 * workload's parameters (cellsize set); nPts, the bounding box and block
 * coordinates, Volume, ParticleVolume, ParticleMass and the indenter
 * position are set here. soa (may be NULL): 16 rows of the pitch
 * oracle_pitch_elems(nPts) doubles. Returns the number of points or -1. */
long oracle_scene_block(icy_SimParams *P, int cells_x, int cells_y, double ind_y_above_floor, double grain_size,
                        uint64_t seed, double *soa)
{
    const double h = P->cellsize;
    if (!(h > 0) || cells_x <= 0 || cells_y <= 0) return -1;
    const long n = 4L * cells_x * cells_y;
    raw_point_t *pts = (raw_point_t *)malloc(sizeof(raw_point_t) * (size_t)n);
    if (!pts) return -1;
    mt64_t *g = (mt64_t *)malloc(sizeof(mt64_t));
    mt64_seed(g, seed);
    long k = 0;
    for (int cy = 0; cy < cells_y; cy++)
        for (int cx = 0; cx < cells_x; cx++)
            for (int sy = 0; sy < 2; sy++)
                for (int sx = 0; sx < 2; sx++) {
                    double jx = (u01(g) - 0.5) * 0.5;
                    double jy = (u01(g) - 0.5) * 0.5;
                    double x = (cx + (sx + 0.5 + jx) * 0.5) * h;
                    double y = (cy + (sy + 0.5 + jy) * 0.5) * h;
                    pts[k].x = (float)x;
                    pts[k].y = (float)y;
                    pts[k].g = 0;
                    pts[k].order = (int)k;
                    k++;
                }

    /* Voronoi grains */
    const double W = cells_x * h, Hb = cells_y * h;
    const double gs = grain_size > 0 ? grain_size : 0.05;
    long ng = lround(W * Hb / (gs * gs));
    if (ng < 1) ng = 1;
    if (ng > 32767) ng = 32767;
    double *sxs = (double *)malloc(sizeof(double) * (size_t)ng), *sys = (double *)malloc(sizeof(double) * (size_t)ng);
    for (long i = 0; i < ng; i++) {
        sxs[i] = u01(g) * W;
        sys[i] = u01(g) * Hb;
    }
    const int bx = imax(1, (int)ceil(W / gs)), by = imax(1, (int)ceil(Hb / gs));
    int *bcount = (int *)calloc((size_t)bx * by + 1, sizeof(int));
    int *bstart = (int *)calloc((size_t)bx * by + 1, sizeof(int));
    int *bitems = (int *)malloc(sizeof(int) * (size_t)ng);
#define BXI(xv) imin(bx - 1, imax(0, (int)((xv) / gs)))
#define BYI(yv) imin(by - 1, imax(0, (int)((yv) / gs)))
    for (long i = 0; i < ng; i++) bcount[BYI(sys[i]) * bx + BXI(sxs[i])]++;
    for (int b = 0; b < bx * by; b++) bstart[b + 1] = bstart[b] + bcount[b];
    memset(bcount, 0, sizeof(int) * (size_t)bx * by);
    for (long i = 0; i < ng; i++) { /* seeds in index order inside each bucket */
        int b = BYI(sys[i]) * bx + BXI(sxs[i]);
        bitems[bstart[b] + bcount[b]++] = (int)i;
    }
    for (long p = 0; p < n; p++) {
        const int cx = BXI(pts[p].x), cy = BYI(pts[p].y);
        double best = 1e300;
        int arg = 0;
        for (int ring = 0; ring <= imax(bx, by); ring++) {
            for (int yy = cy - ring; yy <= cy + ring; yy++)
                for (int xx = cx - ring; xx <= cx + ring; xx++) {
                    if (xx < 0 || yy < 0 || xx >= bx || yy >= by) continue;
                    if (imax(abs(xx - cx), abs(yy - cy)) != ring) continue;
                    const int b = yy * bx + xx;
                    for (int q = bstart[b]; q < bstart[b + 1]; q++) {
                        const int s = bitems[q];
                        double dx = sxs[s] - pts[p].x, dy = sys[s] - pts[p].y;
                        double dd = dx * dx + dy * dy;
                        if (dd < best || (dd == best && s < arg)) {
                            best = dd;
                            arg = s;
                        }
                    }
                }
            if (best < 1e300 && sqrt(best) <= ring * gs) break;
        }
        pts[p].g = (short)arg;
    }
#undef BXI
#undef BYI
    free(bcount);
    free(bstart);
    free(bitems);
    free(sxs);
    free(sys);
    free(g);

    /* SortPoints (stable: equal keys keep the input order) */
    if (P->SortPointsByGridCell) {
        const double hinv = P->cellsize_inv;
        for (long p = 0; p < n; p++)
            pts[p].key = (int)(pts[p].x * hinv - 0.5) + ((int)(pts[p].y * hinv - 0.5)) * P->GridX;
        qsort(pts, (size_t)n, sizeof(raw_point_t), cmp_key);
    }

    /* bounding box, block coordinates, placement */
    P->nPts = (int)n;
    float xmn = pts[0].x, xmx = pts[0].x, ymn = pts[0].y, ymx = pts[0].y;
    for (long p = 1; p < n; p++) {
        if (pts[p].x < xmn) xmn = pts[p].x;
        if (pts[p].x > xmx) xmx = pts[p].x;
        if (pts[p].y < ymn) ymn = pts[p].y;
        if (pts[p].y > ymx) ymx = pts[p].y;
    }
    P->xmin = xmn;
    P->xmax = xmx;
    P->ymin = ymn;
    P->ymax = ymx;
    const float length = (float)(P->xmax - P->xmin);
    P->nxmin = (int)floor(P->xmin / P->cellsize);
    P->nxmax = (int)ceil(P->xmax / P->cellsize);
    P->nymin = (int)floor(P->ymin / P->cellsize);
    P->nymax = (int)ceil(P->ymax / P->cellsize);
    const double x_offset = (P->GridX * h - length) / 2, y_offset = 2 * h;
    P->Volume = (double)(float)(W * Hb);
    const double r = P->IndDiameter / 2;
    P->indenter_x = P->xmin + x_offset - r;
    P->indenter_y = P->ymin + y_offset + ind_y_above_floor;
    P->indenter_x_initial = P->indenter_x;
    P->indenter_y_initial = P->indenter_y;
    P->ParticleVolume = P->Volume / (double)n;
    P->ParticleMass = P->ParticleVolume * P->Density;

    if (soa) {
        const size_t pitch = ((size_t)n + 63) / 64 * 64;
        memset(soa, 0, sizeof(double) * pitch * ICM_N_PTS_ARRAYS);
        uint8_t *crushed = (uint8_t *)soa;
        short *grain = (short *)((char *)soa + pitch);
        for (long p = 0; p < n; p++) {
            float fx = (float)(pts[p].x + x_offset), fy = (float)(pts[p].y + y_offset);
            crushed[p] = 0;
            grain[p] = pts[p].g;
            soa[(size_t)ICM_IDX_JP_INV * pitch + p] = 1.0;
            soa[(size_t)ICM_IDX_POSX * pitch + p] = fx;
            soa[(size_t)(ICM_IDX_POSX + 1) * pitch + p] = fy;
            soa[(size_t)ICM_IDX_FE00 * pitch + p] = 1.0;
            soa[(size_t)(ICM_IDX_FE00 + 3) * pitch + p] = 1.0;
        }
    }
    free(pts);
    return n;
}
