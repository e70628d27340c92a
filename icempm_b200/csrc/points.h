// points.h -- the point pipeline of SnapshotManager::LoadRawPoints
// (simulation/snapshotmanager.cpp:186-286), shared by the raw-point loader
// and the synthetic block: float32 raw points sorted by grid cell with the
// SortPoints key (:288-304; a stable sort here, so equal keys keep input
// order), bounding box and integer block coordinates (:229-240), the block
// centred in x and lifted by 2h (:244-250), and the SoA fill of
// Point::Reset + TransferToBuffer (point.cpp:8-37) with positions offset in
// float arithmetic (:275-276) and widened to double.
#pragma once
#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/icempm.h"

namespace icm {

struct RawPoint { float x, y; short g; };

inline void sort_points(const icy_SimParams &p, std::vector<RawPoint> &pts)
{
    const double hinv = p.cellsize_inv;
    const int gx = p.GridX;
    std::stable_sort(pts.begin(), pts.end(), [hinv, gx](const RawPoint &a, const RawPoint &b) {
        int ai = (int)(a.x * hinv - 0.5) + ((int)(a.y * hinv - 0.5)) * gx;
        int bi = (int)(b.x * hinv - 0.5) + ((int)(b.y * hinv - 0.5)) * gx;
        return ai < bi;
    });
}

struct Placement { double x_offset, y_offset; };

// Sets nPts, the bounding box and block coordinates; returns the offsets
// that place the block (Volume, indenter and particle mass are the
// caller's).
inline Placement place_points(icy_SimParams *p, const std::vector<RawPoint> &pts)
{
    p->nPts = (int)pts.size();
    auto mmx = std::minmax_element(pts.begin(), pts.end(), [](const RawPoint &a, const RawPoint &b) { return a.x < b.x; });
    p->xmin = mmx.first->x;
    p->xmax = mmx.second->x;
    const float length = (float)(p->xmax - p->xmin);
    auto mmy = std::minmax_element(pts.begin(), pts.end(), [](const RawPoint &a, const RawPoint &b) { return a.y < b.y; });
    p->ymin = mmy.first->y;
    p->ymax = mmy.second->y;
    icm_params_compute_block_coords(p);
    const double h = p->cellsize;
    const double box_x = p->GridX * h;
    return {(box_x - length) / 2, 2 * h};
}

inline void fill_soa(const std::vector<RawPoint> &pts, const Placement &pl, double *host_soa, size_t pitch)
{
    const size_t n = pts.size();
    std::memset(host_soa, 0, sizeof(double) * pitch * ICM_N_PTS_ARRAYS);
    uint8_t *crushed = (uint8_t *)host_soa;
    short *grain = (short *)((char *)host_soa + pitch);
    for (size_t i = 0; i < n; i++) {
        float fx = pts[i].x, fy = pts[i].y;
        fx = (float)(fx + pl.x_offset);
        fy = (float)(fy + pl.y_offset);
        crushed[i] = 0;
        grain[i] = pts[i].g;
        host_soa[(size_t)ICM_IDX_JP_INV * pitch + i] = 1.0;
        host_soa[(size_t)ICM_IDX_POSX * pitch + i] = fx;
        host_soa[(size_t)(ICM_IDX_POSX + 1) * pitch + i] = fy;
        host_soa[(size_t)ICM_IDX_FE00 * pitch + i] = 1.0;
        host_soa[(size_t)(ICM_IDX_FE00 + 3) * pitch + i] = 1.0;
    }
}

}  // namespace icm
