// scene.cpp -- seeded synthetic ice block, standing in for
// SnapshotManager::LoadRawPoints (simulation/snapshotmanager.cpp:186-286)
// when no HDF5 point cloud is used.
//
// The point pipeline of LoadRawPoints is kept (points.h): float32 raw
// points, sorted by grid cell, centred in x and lifted by 2h in float
// arithmetic, then widened to double. Volume = block area, ParticleVolume =
// Volume/N and ParticleMass = rho * ParticleVolume follow :225-242 and
// :267-268.
// Deviation (documented): the indenter starts just touching the block's left
// face, x = block_left - r, at an explicit height above the block bottom,
// instead of the IndDepth-based placement of :253-265.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>
#include <vector>

#include "../../include/icempm.h"
#include "errors.h"
#include "points.h"

namespace {

inline double u01(std::mt19937_64 &g) { return (double)(g() >> 11) * (1.0 / 9007199254740992.0); }

}  // namespace

extern "C" int icm_scene_block(icy_SimParams *p, const icm_block_desc *d, double *host_soa, int *n_out)
{
    if (!p || !d) return icm::fail(ICM_ERR_ARG, "icm_scene_block: null argument");
    if (d->cells_x <= 0 || d->cells_y <= 0) return icm::fail(ICM_ERR_ARG, "icm_scene_block: empty block");
    const double h = p->cellsize;
    if (!(h > 0)) return icm::fail(ICM_ERR_STATE, "icm_scene_block: cellsize not set (parse or reset params first)");
    const long n = 4L * d->cells_x * d->cells_y;
    if (n > 0x7fffffffL) return icm::fail(ICM_ERR_ARG, "icm_scene_block: too many particles");
    if (n_out) *n_out = (int)n;

    std::mt19937_64 rng(d->seed);
    std::vector<icm::RawPoint> pts((size_t)n);
    size_t k = 0;
    for (int cy = 0; cy < d->cells_y; cy++)
        for (int cx = 0; cx < d->cells_x; cx++)
            for (int sy = 0; sy < 2; sy++)
                for (int sx = 0; sx < 2; sx++) {
                    double jx = (u01(rng) - 0.5) * 0.5, jy = (u01(rng) - 0.5) * 0.5;  // +-0.25 sub-cell
                    double x = (cx + (sx + 0.5 + jx) * 0.5) * h;
                    double y = (cy + (sy + 0.5 + jy) * 0.5) * h;
                    pts[k++] = {(float)x, (float)y, 0};
                }

    // Voronoi grains
    const double W = d->cells_x * h, Hb = d->cells_y * h;
    const double gs = d->grain_size > 0 ? d->grain_size : 0.05;
    long ng = std::max(1L, std::lround(W * Hb / (gs * gs)));
    if (ng > 32767) ng = 32767;
    std::vector<double> sx((size_t)ng), sy((size_t)ng);
    for (long i = 0; i < ng; i++) {
        sx[(size_t)i] = u01(rng) * W;
        sy[(size_t)i] = u01(rng) * Hb;
    }
    // bucket the seeds on a coarse grid of ~gs cells; search rings until found
    const int bx = std::max(1, (int)std::ceil(W / gs)), by = std::max(1, (int)std::ceil(Hb / gs));
    std::vector<std::vector<int>> bucket((size_t)bx * by);
    auto bxi = [&](double x) { return std::min(bx - 1, std::max(0, (int)(x / gs))); };
    auto byi = [&](double y) { return std::min(by - 1, std::max(0, (int)(y / gs))); };
    for (long i = 0; i < ng; i++) bucket[(size_t)byi(sy[(size_t)i]) * bx + bxi(sx[(size_t)i])].push_back((int)i);
    for (auto &q : pts) {
        int cx = bxi(q.x), cy = byi(q.y);
        double best = 1e300;
        int arg = 0;
        for (int ring = 0; ring <= std::max(bx, by); ring++) {
            for (int yy = cy - ring; yy <= cy + ring; yy++)
                for (int xx = cx - ring; xx <= cx + ring; xx++) {
                    if (xx < 0 || yy < 0 || xx >= bx || yy >= by) continue;
                    if (std::max(std::abs(xx - cx), std::abs(yy - cy)) != ring) continue;
                    for (int s : bucket[(size_t)yy * bx + xx]) {
                        double dx = sx[(size_t)s] - q.x, dy = sy[(size_t)s] - q.y;
                        double dd = dx * dx + dy * dy;
                        if (dd < best || (dd == best && s < arg)) {
                            best = dd;
                            arg = s;
                        }
                    }
                }
            // every seed outside this ring is at least ring*gs away
            if (best < 1e300 && std::sqrt(best) <= ring * gs) break;
        }
        q.g = (short)arg;
    }

    if (p->SortPointsByGridCell) icm::sort_points(*p, pts);

    const icm::Placement pl = icm::place_points(p, pts);
    p->Volume = (double)(float)(W * Hb);
    const double r = p->IndDiameter / 2;
    const double block_left = p->xmin + pl.x_offset;
    const double block_bottom = p->ymin + pl.y_offset;
    p->indenter_x = block_left - r;
    p->indenter_y = block_bottom + d->ind_y_above_floor;
    p->indenter_x_initial = p->indenter_x;
    p->indenter_y_initial = p->indenter_y;
    p->ParticleVolume = p->Volume / (double)n;
    p->ParticleMass = p->ParticleVolume * p->Density;

    if (host_soa) icm::fill_soa(pts, pl, host_soa, icm_pitch_elems((size_t)n));
    return ICM_OK;
}
