/*
 * icempm.hpp -- header-only C++ face of libicempm.so with the names of
 * iceMPM's device layer, so that code written against
 * simulation/gpu_implementation5.h, simulation/model.h,
 * simulation/parameters_sim.h and simulation/point.h compiles against it
 * (Eigen types excepted: positions come back as std::array<double, 2>).
 *
 *   icy::SimParams       parameters_sim.h:17-90 (same 432-byte layout; the
 *                        methods call icm_params_*)
 *   icy::Point           point.h:14-37, the static SoA accessors
 *   GPU_Implementation5  gpu_implementation5.h:40-72; every member forwards
 *                        to the C ABI and throws std::runtime_error with
 *                        icm_last_error() on a non-zero status, as the
 *                        reference members throw on CUDA errors
 *   icy::Model           model.h:26-52, model.cpp:11-67
 *   icy::SnapshotManager snapshotmanager.h:15-31 (HDF5 without libhdf5)
 *
 * Extensions (no counterpart in the reference): GPU_Implementation5::
 * set_form / set_tile / run_substeps select and run the fused forms;
 * icy::Model::Step runs a frame through run_substeps.
 *
 * Link with -licempm; the CUDA headers are not needed.
 */
#ifndef ICEMPM_HPP
#define ICEMPM_HPP

#include <array>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <functional>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "icempm.h"

/* cudaEvent_t as cuda_runtime_api.h declares it (an identical typedef may
 * appear in both). */
struct CUevent_st;
typedef struct CUevent_st *cudaEvent_t;

namespace icy {

inline void icm_check(int rc)
{
    if (rc != ICM_OK) throw std::runtime_error(icm_last_error());
}

struct SimParams : icy_SimParams {
    constexpr static size_t idx_utility_data = ICM_IDX_UTILITY;
    constexpr static size_t idx_P = ICM_IDX_P;
    constexpr static size_t idx_Q = ICM_IDX_Q;
    constexpr static size_t idx_Jp_inv = ICM_IDX_JP_INV;
    constexpr static size_t posx = ICM_IDX_POSX;
    constexpr static size_t velx = ICM_IDX_VELX;
    constexpr static size_t Fe00 = ICM_IDX_FE00;
    constexpr static size_t Bp00 = ICM_IDX_BP00;
    constexpr static size_t nPtsArrays = ICM_N_PTS_ARRAYS;
    constexpr static size_t nGridArrays = ICM_N_GRID_ARRAYS;

    void Reset() { icm_params_reset(this); }
    /* Returns the raw-points file named by the configuration ("" when none). */
    std::string ParseFile(std::string fileName)
    {
        char raw[4096] = {0};
        icm_check(icm_params_parse_file(this, fileName.c_str(), raw, sizeof(raw)));
        return std::string(raw);
    }
    void ComputeLame() { icm_params_compute_lame(this); }
    void ComputeCamClayParams2() { icm_params_compute_camclay(this); }
    void ComputeHelperVariables() { icm_params_compute_helpers(this); }
    void ComputeIntegerBlockCoords() { icm_params_compute_block_coords(this); }
    size_t IndenterArraySize() const { return sizeof(double) * 2 * (size_t)n_indenter_subdivisions; }
};
static_assert(sizeof(SimParams) == sizeof(icy_SimParams), "SimParams must keep the 432-byte layout");

/* Static accessors of the pitched particle SoA (point.cpp:39-70). */
struct Point {
    static std::array<double, 2> getPos(const double *buffer, const int pitch, const int i)
    {
        return {buffer[i + pitch * SimParams::posx], buffer[i + pitch * (SimParams::posx + 1)]};
    }
    static uint8_t getCrushedStatus(const double *buffer, const int pitch, const int i)
    {
        return reinterpret_cast<const uint8_t *>(buffer + pitch * SimParams::idx_utility_data)[i];
    }
    static double getJp_inv(const double *buffer, const int pitch, const int i)
    {
        return buffer[i + pitch * SimParams::idx_Jp_inv];
    }
    static short getGrain(const double *buffer, const int pitch, const int i)
    {
        short g;
        std::memcpy(&g, reinterpret_cast<const char *>(buffer + pitch * SimParams::idx_utility_data) +
                            sizeof(double) * pitch + sizeof(short) * (size_t)i, sizeof(short));
        return g;
    }
    static std::pair<double, double> getPQ(const double *buffer, const int pitch, const int i)
    {
        return {buffer[i + pitch * SimParams::idx_P], buffer[i + pitch * SimParams::idx_Q]};
    }
};

/* The cycle lock of model.h:42. The simulation thread takes it before a
 * frame's copy to the host and the thread that consumes the frame releases
 * it (cli/main.cpp:51-62), so it is a binary semaphore rather than a
 * std::mutex, which the locking thread alone may unlock. */
class CycleLock {
public:
    void lock()
    {
        std::unique_lock<std::mutex> l(m_);
        cv_.wait(l, [&] { return !held_; });
        held_ = true;
    }
    void unlock()
    {
        {
            std::lock_guard<std::mutex> l(m_);
            held_ = false;
        }
        cv_.notify_all();
    }

private:
    std::mutex m_;
    std::condition_variable cv_;
    bool held_ = false;
};

class Model;

}  // namespace icy

class GPU_Implementation5 {
public:
    icy::Model *model = nullptr;
    int error_code = 0;
    std::function<void()> transfer_completion_callback;

    cudaEvent_t eventCycleStart = nullptr, eventCycleStop = nullptr;

    double *tmp_transfer_buffer = nullptr;  // pinned host mirror of the particle SoA
    double *host_side_indenter_force_accumulator = nullptr;

    GPU_Implementation5() = default;
    GPU_Implementation5(const GPU_Implementation5 &) = delete;
    GPU_Implementation5 &operator=(const GPU_Implementation5 &) = delete;
    ~GPU_Implementation5()
    {
        if (ctx_) icm_destroy(ctx_);
        if (tmp_transfer_buffer) icm_host_free(tmp_transfer_buffer);
        if (host_side_indenter_force_accumulator) icm_host_free(host_side_indenter_force_accumulator);
    }

    void initialize()
    {
        if (ctx_) return;
        icy::icm_check(icm_create(&ctx_, 0));
        void *a = nullptr, *b = nullptr;
        icy::icm_check(icm_cycle_events(ctx_, &a, &b));
        eventCycleStart = static_cast<cudaEvent_t>(a);
        eventCycleStop = static_cast<cudaEvent_t>(b);
    }
    void test() {}
    void synchronize()
    {
        if (ctx_) icy::icm_check(icm_synchronize(ctx_));
    }
    inline void cuda_update_constants();
    inline void cuda_allocate_arrays(size_t nGridNodes, size_t nPoints);
    void cuda_reset_grid() { icy::icm_check(icm_reset_grid(ctx_)); }
    inline void transfer_ponts_to_device();
    void cuda_p2g() { icy::icm_check(icm_p2g(ctx_)); }
    void cuda_g2p(bool recordPQ) { icy::icm_check(icm_g2p(ctx_, recordPQ ? 1 : 0)); }
    void cuda_update_nodes(double indenter_x, double indenter_y)
    {
        icy::icm_check(icm_update_nodes(ctx_, indenter_x, indenter_y));
    }
    void cuda_reset_indenter_force_accumulator() { icy::icm_check(icm_reset_indenter_force_accumulator(ctx_)); }
    void cuda_transfer_from_device()
    {
        icy::icm_check(icm_transfer_from_device(ctx_, tmp_transfer_buffer, host_side_indenter_force_accumulator,
                                                &error_code, &GPU_Implementation5::callback_from_stream, this));
    }

    // extensions
    void set_form(int form)
    {
        initialize();
        icy::icm_check(icm_set_form(ctx_, form));
    }
    void set_tile(int variant, int threads)
    {
        initialize();
        icy::icm_check(icm_set_tile(ctx_, variant, threads));
    }
    inline void run_substeps(int n);
    void run_substeps(icy_SimParams &p, int n) { icy::icm_check(icm_run_substeps(ctx_, &p, n)); }
    void set_rebin_interval(int substeps)
    {
        initialize();
        icy::icm_check(icm_set_rebin_interval(ctx_, substeps));
    }
    void set_tile_split(int max_tiles, double ratio)
    {
        initialize();
        icy::icm_check(icm_set_tile_split(ctx_, max_tiles, ratio));
    }
    icm_ctx *context() const { return ctx_; }

private:
    icm_ctx *ctx_ = nullptr;
    static void callback_from_stream(void *user)
    {
        auto *gpu = static_cast<GPU_Implementation5 *>(user);
        if (gpu->transfer_completion_callback) gpu->transfer_completion_callback();
    }
};

class icy::Model {
public:
    Model()
    {
        prms.Reset();
        gpu.model = this;
    }
    void Reset()
    {
        prms.SimulationStep = 0;
        prms.SimulationTime = 0;
        compute_time_per_cycle = 0;
    }
    void Prepare()
    {
        abortRequested = false;
        gpu.cuda_update_constants();
    }
    /* One frame: the substeps up to the next multiple of UpdateEveryNthStep
     * (model.cpp:11-47), run on the device in the form set on gpu, then the
     * asynchronous D2H copy and callback. Returns false at the end time or
     * after an out-of-grid error. */
    bool Step()
    {
        const int n = prms.UpdateEveryNthStep - prms.SimulationStep % prms.UpdateEveryNthStep;
        const bool timed = prms.SimulationStep % (prms.UpdateEveryNthStep * 2) == 0;
        gpu.cuda_reset_indenter_force_accumulator();
        if (timed) icm_check(icm_record_start(gpu.context()));
        // the frame advances a copy: the consumer of the previous frame may
        // still read prms until the cycle lock is ours (model.cpp:32-45
        // updates them after taking it)
        icy_SimParams next = prms;
        gpu.run_substeps(next, n);
        if (timed) icm_check(icm_record_stop(gpu.context()));
        processing_current_cycle_data.lock();  // held until the host has consumed the frame
        prms.SimulationStep = next.SimulationStep;
        prms.SimulationTime = next.SimulationTime;
        prms.indenter_x = next.indenter_x;
        gpu.cuda_transfer_from_device();
        if (!timed) {
            float ms = 0;
            if (icm_elapsed_ms(gpu.context(), &ms) == ICM_OK) compute_time_per_cycle = ms / prms.UpdateEveryNthStep;
        }
        return prms.SimulationTime < prms.SimulationEndTime && !gpu.error_code;
    }
    void RequestAbort() { abortRequested = true; }
    void UnlockCycleMutex() { processing_current_cycle_data.unlock(); }

    icy::SimParams prms;
    GPU_Implementation5 gpu;
    float compute_time_per_cycle = 0;
    icy::CycleLock processing_current_cycle_data;

private:
    bool abortRequested = false;
};

namespace icy {
/* Many cases advanced together, one launch per substep for all of them
 * (icm_ensemble_*); no counterpart in the reference, which runs one case per
 * process. Each case is a Model set up as for Step (block loaded, constants
 * updated); run(n) advances every case n substeps and leaves its results
 * in the case, as GPU_Implementation5::run_substeps would. */
class Ensemble {
public:
    explicit Ensemble(int form = ICM_FORM_FP32, int tile_variant = 1, int threads = 128, int device = 0)
    {
        icm_check(icm_ensemble_create(&e_, device, form, tile_variant, threads));
    }
    Ensemble(const Ensemble &) = delete;
    Ensemble &operator=(const Ensemble &) = delete;
    ~Ensemble()
    {
        if (e_) icm_ensemble_destroy(e_);
    }
    void add(Model &m)
    {
        m.gpu.initialize();
        icm_check(icm_ensemble_add(e_, m.gpu.context()));
        cases_.push_back(&m);
    }
    void set(int rebin_interval, bool graphs = true) { icm_check(icm_ensemble_set(e_, rebin_interval, graphs ? 1 : 0)); }
    void set_split(int max_tiles, double ratio) { icm_check(icm_ensemble_set_split(e_, max_tiles, ratio)); }
    void run(int n)
    {
        std::vector<icy_SimParams *> p;
        for (Model *m : cases_) p.push_back(&m->prms);
        icm_check(icm_ensemble_run(e_, p.data(), n));
    }
    void synchronize()
    {
        for (Model *m : cases_) m->gpu.synchronize();
    }
    void *stream() const { return icm_ensemble_stream(e_); }
    size_t size() const { return cases_.size(); }

private:
    icm_ensemble *e_ = nullptr;
    std::vector<Model *> cases_;
};
}  // namespace icy

/* icy::SnapshotManager (snapshotmanager.h:15-31) over the library's HDF5
 * code. ReadSnapshot resumes a run (the reference's is commented out). */
namespace icy {
class SnapshotManager {
public:
    icy::Model *model = nullptr;
    const std::string directory_snapshots = "snapshots";
    const std::string directory_pq = "pq";

    std::string SaveSnapshot(std::string outputDirectory)
    {
        char path[4096];
        icm_check(icm_save_snapshot(&model->prms, model->gpu.tmp_transfer_buffer,
                                    model->gpu.host_side_indenter_force_accumulator, outputDirectory.c_str(), path,
                                    sizeof(path)));
        return path;
    }
    std::string SavePQ(std::string outputDirectory)
    {
        char path[4096];
        icm_check(icm_save_pq(&model->prms, model->gpu.tmp_transfer_buffer, outputDirectory.c_str(), path,
                              sizeof(path)));
        return path;
    }
    void LoadRawPoints(std::string fileName)
    {
        int n = 0;
        icm_check(icm_load_raw_points(&model->prms, fileName.c_str(), nullptr, &n));
        model->gpu.cuda_allocate_arrays((size_t)model->prms.GridX * model->prms.GridY, (size_t)n);
        icm_check(icm_load_raw_points(&model->prms, fileName.c_str(), model->gpu.tmp_transfer_buffer, &n));
        model->gpu.transfer_ponts_to_device();
        model->Reset();
        model->Prepare();
    }
    /* Returns the frame number of the snapshot. */
    int ReadSnapshot(std::string fileName)
    {
        icy_SimParams tmp;
        icm_check(icm_read_snapshot_params(fileName.c_str(), &tmp));
        const size_t src_pitch = tmp.nPtsPitch, n = (size_t)tmp.nPts;
        std::vector<double> soa(src_pitch * SimParams::nPtsArrays), bins(2 * (size_t)tmp.n_indenter_subdivisions);
        icm_check(icm_read_snapshot(fileName.c_str(), soa.data(), soa.size(), bins.data(), bins.size()));
        SimParams &p = model->prms;
        const bool realloc = !model->gpu.tmp_transfer_buffer || tmp.nPts > p.nPts ||
                             (size_t)tmp.GridX * tmp.GridY > (size_t)p.GridX * p.GridY ||
                             tmp.n_indenter_subdivisions != p.n_indenter_subdivisions;
        icy_SimParams keep = p;
        static_cast<icy_SimParams &>(p) = tmp;
        if (realloc) {
            model->gpu.cuda_allocate_arrays((size_t)tmp.GridX * tmp.GridY, n);
        } else {
            p.grid_array = keep.grid_array;
            p.pts_array = keep.pts_array;
            p.indenter_force_accumulator = keep.indenter_force_accumulator;
            p.nPtsPitch = keep.nPtsPitch;
            p.nGridPitch = keep.nGridPitch;
        }
        // the utility row holds crushed bytes at byte i and grain ids at
        // byte pitch + 2i (point.cpp:19-23): move it field by field
        const size_t dst_pitch = p.nPtsPitch;
        double *dst = model->gpu.tmp_transfer_buffer;
        std::memset(dst, 0, sizeof(double) * dst_pitch * SimParams::nPtsArrays);
        for (size_t r = 1; r < SimParams::nPtsArrays; r++)
            std::memcpy(dst + r * dst_pitch, soa.data() + r * src_pitch, sizeof(double) * n);
        const char *s0 = reinterpret_cast<const char *>(soa.data());
        char *d0 = reinterpret_cast<char *>(dst);
        std::memcpy(d0, s0, n);
        std::memcpy(d0 + dst_pitch, s0 + src_pitch, 2 * n);
        model->gpu.transfer_ponts_to_device();
        std::memcpy(model->gpu.host_side_indenter_force_accumulator, bins.data(), sizeof(double) * bins.size());
        model->Prepare();
        return p.UpdateEveryNthStep > 0 ? p.SimulationStep / p.UpdateEveryNthStep : 0;
    }
};
}  // namespace icy

inline void GPU_Implementation5::cuda_update_constants()
{
    icy::icm_check(icm_update_constants(ctx_, &model->prms, error_code));
}

inline void GPU_Implementation5::cuda_allocate_arrays(size_t nGridNodes, size_t nPoints)
{
    initialize();
    if (tmp_transfer_buffer) icm_host_free(tmp_transfer_buffer);
    if (host_side_indenter_force_accumulator) icm_host_free(host_side_indenter_force_accumulator);
    tmp_transfer_buffer = nullptr;
    host_side_indenter_force_accumulator = nullptr;
    icy::icm_check(icm_allocate_arrays(ctx_, &model->prms, nGridNodes, nPoints));
    void *a = nullptr, *b = nullptr;
    icy::icm_check(icm_host_alloc(&a, sizeof(double) * model->prms.nPtsPitch * icy::SimParams::nPtsArrays));
    tmp_transfer_buffer = static_cast<double *>(a);
    icy::icm_check(icm_host_alloc(&b, model->prms.IndenterArraySize()));
    host_side_indenter_force_accumulator = static_cast<double *>(b);
    error_code = 0;
}

inline void GPU_Implementation5::transfer_ponts_to_device()
{
    icy::icm_check(icm_transfer_points_to_device(ctx_, tmp_transfer_buffer));
    std::memset(host_side_indenter_force_accumulator, 0, model->prms.IndenterArraySize());
}

inline void GPU_Implementation5::run_substeps(int n)
{
    icy::icm_check(icm_run_substeps(ctx_, &model->prms, n));
}

#endif /* ICEMPM_HPP */
