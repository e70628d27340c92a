// snapshot.cpp -- SnapshotManager (simulation/snapshotmanager.cpp) on the
// library's own HDF5 writer and reader (hdf5_lite.h): full snapshots
// (SaveSnapshot :60-104, SaveParametersAsAttributes :106-142), reading them
// back to resume a run (the reference's ReadSnapshot :145-184 is commented
// out), P/Q dumps (SavePQ :14-56) and raw point clouds (LoadRawPoints
// :186-286, SortPoints :288-304). Host-side; no CUDA.
#include <cmath>
#include <cstdio>
#include <filesystem>
#include <string>
#include <vector>

#include "../../include/icempm.h"
#include "errors.h"
#include "hdf5_lite.h"
#include "points.h"

namespace {

int put_path(const std::string &path, char *out, size_t cap)
{
    if (out && cap) {
        if (path.size() + 1 > cap) return icm::fail(ICM_ERR_ARG, "path buffer too small for " + path);
        std::memcpy(out, path.c_str(), path.size() + 1);
    }
    return ICM_OK;
}

int frame_number(const icy_SimParams *p) { return p->UpdateEveryNthStep > 0 ? p->SimulationStep / p->UpdateEveryNthStep : 0; }

// <dir>/<sub>/<prefix>NNNNN.h5, creating the directories
int frame_path(const char *dir, const char *sub, const char *prefix, int frame, std::string &path)
{
    char name[32];
    std::snprintf(name, sizeof(name), "%s%05d.h5", prefix, frame);
    std::error_code ec;
    const std::filesystem::path d = std::filesystem::path(dir) / sub;
    std::filesystem::create_directories(d, ec);
    if (ec) return icm::fail(ICM_ERR_IO, "cannot create directory " + d.string() + ": " + ec.message());
    path = (d / name).string();
    return ICM_OK;
}

// SaveParametersAsAttributes (snapshotmanager.cpp:106-142), same names,
// types and order
std::vector<h5l::Attr> parameter_attrs(const icy_SimParams *p)
{
    using namespace h5l;
    return {attr("indenter_x", f64(), p->indenter_x),
            attr("indenter_y", f64(), p->indenter_y),
            attr("SimulationTime", f64(), p->SimulationTime),
            attr("GridX", i32(), (int32_t)p->GridX),
            attr("GridY", i32(), (int32_t)p->GridY),
            attr("nPts", i32(), (int32_t)p->nPts),
            attr("nPtsPitch", i64(), (int64_t)p->nPtsPitch),
            attr("UpdateEveryNthStep", i32(), (int32_t)p->UpdateEveryNthStep),
            attr("n_indenter_subdivisions", i32(), (int32_t)p->n_indenter_subdivisions),
            attr("cellsize", f64(), p->cellsize),
            attr("IndDiameter", f64(), p->IndDiameter),
            attr("InitialTimeStep", f64(), p->InitialTimeStep),
            attr("SetupType", i32(), (int32_t)p->SetupType),
            attr("Volume", f64(), p->Volume)};
}

bool same_type(const h5l::Type &a, const h5l::Type &b) { return a.cls == b.cls && a.size == b.size; }

}  // namespace

extern "C" int icm_save_snapshot(const icy_SimParams *p, const double *host_soa, const double *host_bins,
                                 const char *dir, char *path_out, size_t cap)
{
    if (!p || !host_soa || !host_bins || !dir) return icm::fail(ICM_ERR_ARG, "icm_save_snapshot: null argument");
    if (p->nPtsPitch < (size_t)p->nPts || p->n_indenter_subdivisions < 1)
        return icm::fail(ICM_ERR_ARG, "icm_save_snapshot: pitch/subdivisions not set");
    std::string path;
    int rc = frame_path(dir, "snapshots", "d", frame_number(p), path);
    if (rc) return rc;
    std::vector<h5l::DatasetSpec> ds(3);
    ds[0] = {"Indenter_2D", h5l::f64(), {2 * (uint64_t)p->n_indenter_subdivisions}, host_bins, {}};
    ds[1] = {"Params", h5l::b8(), {sizeof(icy_SimParams)}, p, parameter_attrs(p)};
    ds[2] = {"Points", h5l::f64(), {(uint64_t)p->nPtsPitch * ICM_N_PTS_ARRAYS}, host_soa, {}};
    const std::string e = h5l::write_file(path, ds);
    if (!e.empty()) return icm::fail(ICM_ERR_IO, "icm_save_snapshot: " + e);
    return put_path(path, path_out, cap);
}

extern "C" int icm_read_snapshot_params(const char *path, icy_SimParams *out)
{
    if (!path || !out) return icm::fail(ICM_ERR_ARG, "icm_read_snapshot_params: null argument");
    h5l::File f;
    std::string e = f.open(path);
    h5l::File::Info in;
    if (e.empty()) e = f.info("Params", in);
    if (!e.empty()) return icm::fail(ICM_ERR_IO, "icm_read_snapshot_params: " + e);
    if (in.dims.size() != 1 || in.dims[0] != sizeof(icy_SimParams) || in.type.size != 1)
        return icm::fail(ICM_ERR_PARSE, "icm_read_snapshot_params: SimParams size mismatch");
    e = f.read("Params", out, sizeof(icy_SimParams));
    if (!e.empty()) return icm::fail(ICM_ERR_IO, "icm_read_snapshot_params: " + e);
    return ICM_OK;
}

extern "C" int icm_read_snapshot(const char *path, double *host_soa, size_t soa_elems, double *host_bins,
                                 size_t bins_elems)
{
    if (!path || !host_soa) return icm::fail(ICM_ERR_ARG, "icm_read_snapshot: null argument");
    h5l::File f;
    std::string e = f.open(path);
    h5l::File::Info pts, ind;
    if (e.empty()) e = f.info("Points", pts);
    if (e.empty()) e = f.info("Indenter_2D", ind);
    if (!e.empty()) return icm::fail(ICM_ERR_IO, "icm_read_snapshot: " + e);
    if (!same_type(pts.type, h5l::f64()) || pts.dims.size() != 1 || pts.dims[0] != soa_elems)
        return icm::fail(ICM_ERR_ARG, "icm_read_snapshot: Points size differs from the buffer (16 x nPtsPitch)");
    e = f.read("Points", host_soa, sizeof(double) * soa_elems);
    if (e.empty() && host_bins) {
        if (!same_type(ind.type, h5l::f64()) || ind.dims.size() != 1 || ind.dims[0] != bins_elems)
            return icm::fail(ICM_ERR_ARG, "icm_read_snapshot: Indenter_2D size differs from the buffer");
        e = f.read("Indenter_2D", host_bins, sizeof(double) * bins_elems);
    }
    if (!e.empty()) return icm::fail(ICM_ERR_IO, "icm_read_snapshot: " + e);
    return ICM_OK;
}

extern "C" int icm_save_pq(const icy_SimParams *p, const double *host_soa, const char *dir, char *path_out,
                           size_t cap)
{
    if (!p || !host_soa || !dir) return icm::fail(ICM_ERR_ARG, "icm_save_pq: null argument");
    const size_t pitch = p->nPtsPitch, n = (size_t)std::max(p->nPts, 0);
    if (pitch < n) return icm::fail(ICM_ERR_ARG, "icm_save_pq: pitch not set");
    std::string path;
    int rc = frame_path(dir, "pq", "pq", frame_number(p), path);
    if (rc) return rc;
    std::vector<double> crushed, intact;
    const uint8_t *cr = reinterpret_cast<const uint8_t *>(host_soa);
    for (size_t i = 0; i < n; i++) {
        std::vector<double> &b = cr[i] ? crushed : intact;
        b.push_back(host_soa[(size_t)ICM_IDX_P * pitch + i]);
        b.push_back(host_soa[(size_t)ICM_IDX_Q * pitch + i]);
    }
    std::vector<h5l::DatasetSpec> ds(2);
    ds[0] = {"PQ_intact", h5l::f64(), {intact.size() / 2, 2}, intact.data(), parameter_attrs(p)};
    ds[1] = {"PQ_crushed", h5l::f64(), {crushed.size() / 2, 2}, crushed.data(), {}};
    const std::string e = h5l::write_file(path, ds);
    if (!e.empty()) return icm::fail(ICM_ERR_IO, "icm_save_pq: " + e);
    return put_path(path, path_out, cap);
}

extern "C" int icm_load_raw_points(icy_SimParams *p, const char *path, double *host_soa, int *n_out)
{
    if (!p || !path) return icm::fail(ICM_ERR_ARG, "icm_load_raw_points: null argument");
    if (!(p->cellsize > 0)) return icm::fail(ICM_ERR_STATE, "icm_load_raw_points: cellsize not set (parse params first)");
    if (!std::filesystem::exists(path)) return icm::fail(ICM_ERR_IO, "error reading raw points file - no file");
    h5l::File f;
    std::string e = f.open(path);
    h5l::File::Info pi, gi;
    if (e.empty()) e = f.info("Points_Raw_2D", pi);
    if (e.empty()) e = f.info("GrainIDs", gi);
    if (!e.empty()) return icm::fail(ICM_ERR_IO, "icm_load_raw_points: " + e);
    if (pi.dims.size() != 2 || pi.dims[1] != 2 || !same_type(pi.type, h5l::f32()))
        return icm::fail(ICM_ERR_PARSE, "error reading raw points file - dimensions mismatch");
    const uint64_t n = pi.dims[0];
    if (n == 0 || n > 0x7fffffffull) return icm::fail(ICM_ERR_PARSE, "icm_load_raw_points: point count out of range");
    if (gi.dims.size() != 1 || gi.dims[0] != n || gi.type.cls != h5l::kFixed || gi.type.size != 2)
        return icm::fail(ICM_ERR_PARSE, "icm_load_raw_points: GrainIDs must be int16[N]");
    std::vector<float> xy(2 * n);
    std::vector<short> grain(n);
    e = f.read("Points_Raw_2D", xy.data(), sizeof(float) * xy.size());
    if (e.empty()) e = f.read("GrainIDs", grain.data(), sizeof(short) * grain.size());
    h5l::Type vt;
    std::vector<uint8_t> vv;
    if (e.empty()) e = f.read_attr("GrainIDs", "volume", vt, vv);
    if (e.empty() && (!same_type(vt, h5l::f32()) || vv.size() != 4)) e = "attribute volume must be one float";
    if (!e.empty()) return icm::fail(ICM_ERR_IO, "icm_load_raw_points: " + e);
    float volume;
    std::memcpy(&volume, vv.data(), 4);

    std::vector<icm::RawPoint> pts(n);
    for (uint64_t i = 0; i < n; i++) pts[i] = {xy[2 * i], xy[2 * i + 1], grain[i]};
    if (p->SortPointsByGridCell) icm::sort_points(*p, pts);
    p->Volume = (double)volume;
    const icm::Placement pl = icm::place_points(p, pts);
    // indenter start (snapshotmanager.cpp:253-265)
    const double h = p->cellsize;
    const double block_left = pl.x_offset;
    const double block_top = p->ymax + pl.y_offset;
    const double r = p->IndDiameter / 2;
    const double ht = r - p->IndDepth;
    const double x_ind_offset = std::sqrt(r * r - ht * ht);
    p->indenter_x = std::floor((block_left - x_ind_offset) / h) * h;
    if (p->SetupType == 0)
        p->indenter_y = block_top + ht;
    else if (p->SetupType == 1)
        p->indenter_y = std::ceil(block_top / h) * h;
    p->indenter_x_initial = p->indenter_x;
    p->indenter_y_initial = p->indenter_y;
    p->ParticleVolume = p->Volume / (double)n;
    p->ParticleMass = p->ParticleVolume * p->Density;
    if (n_out) *n_out = (int)n;
    if (host_soa) {
        if (p->nPtsPitch < n) return icm::fail(ICM_ERR_STATE, "icm_load_raw_points: allocate arrays before filling");
        icm::fill_soa(pts, pl, host_soa, p->nPtsPitch);
    }
    return ICM_OK;
}
