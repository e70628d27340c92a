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
#include <cstdint>
#include <cstring>
#include <functional>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>

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
        gpu.run_substeps(n);
        if (timed) icm_check(icm_record_stop(gpu.context()));
        processing_current_cycle_data.lock();  // held until the host has consumed the frame
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
    std::mutex processing_current_cycle_data;

private:
    bool abortRequested = false;
};

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
