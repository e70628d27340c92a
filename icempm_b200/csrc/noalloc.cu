// noalloc.cu -- a substep entry point that allocates no memory.
//
// Some callers cannot allocate device memory while they run: an allocator
// call can block or synchronise the whole device, a host framework may own
// every byte of the GPU through its own pool, or the caller runs under a
// fixed memory budget decided up front. icm_run_substeps_noalloc serves
// them: the caller passes its particle buffer and output buffers, and the
// only scratch the substep needs -- the background grid -- lives in one
// file-scope device array of fixed size that every GPU loading this library
// holds until the process exits.
//
// The grid scratch holds at most kNoAllocMaxNodes nodes (GridX * GridY),
// three doubles each: 262,144 nodes, 6 MiB. All calls share it, so calls
// that overlap on the GPU (two streams, two threads) race on the grid and
// must not be issued concurrently. The grid is cleared at the start of every
// substep, so the contents a previous call left behind do not matter.
//
// The kernels are the FP64 step-wise ones of the member-style API
// (k_stepwise.cuh); only the grid they scatter into differs.
#include <cuda_runtime.h>
#include <mutex>
#include <string>

#include "../../include/icempm.h"
#include "errors.h"

namespace icm {
__global__ void k_p2g_ref64(const icy_SimParams P, int *err);
__global__ void k_update_ref64(const icy_SimParams P, double ind_x, double ind_y, double *force_total);
__global__ void k_g2p_ref64(const icy_SimParams P, int recordPQ);
}  // namespace icm

namespace {

constexpr size_t kNoAllocMaxNodes = 262144;
constexpr int kMaxDevices = 64;

// The grid scratch: 3 rows (mass, momentum x | velocity x, momentum y |
// velocity y) of GridX * GridY doubles, packed one after another.
static __device__ __align__(256) double g_noalloc_grid[3 * kNoAllocMaxNodes];

// Device address of g_noalloc_grid per device. In host code the symbol is
// only a host-side stand-in; the kernels must be given this address. It is
// looked up again (cudaGetSymbolAddress, with the device current) on every
// call made outside stream capture, so that a context created anew on the
// device (after cudaDeviceReset, say) gets its own address; a call made
// while its stream is being captured takes the address of the last call on
// the device, which must have come before the capture began.
std::mutex g_setup_mutex;
double *g_grid_addr[kMaxDevices] = {};

int grid_address(cudaStream_t s, double **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return icm::fail(ICM_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return icm::fail(ICM_ERR_ARG, "icm_run_substeps_noalloc: device index too large");
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    e = cudaStreamIsCapturing(s, &cs);
    if (e != cudaSuccess) return icm::fail(ICM_ERR_CUDA, std::string("cudaStreamIsCapturing: ") + cudaGetErrorString(e));
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (cs == cudaStreamCaptureStatusNone) {
        void *ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_grid);
        if (e != cudaSuccess || !ptr)
            return icm::fail(ICM_ERR_CUDA, std::string("cudaGetSymbolAddress(grid scratch): ") + cudaGetErrorString(e));
        g_grid_addr[dev] = static_cast<double *>(ptr);
    } else if (!g_grid_addr[dev]) {
        return icm::fail(ICM_ERR_STATE,
                         "icm_run_substeps_noalloc: the first call on a device must come before any stream capture");
    }
    *out = g_grid_addr[dev];
    return ICM_OK;
}

}  // namespace

extern "C" int icm_run_substeps_noalloc(icy_SimParams *p, double *pts, double *bins, int *err, int n, void *stream)
{
    if (!p || !pts || !bins || !err) return icm::fail(ICM_ERR_ARG, "icm_run_substeps_noalloc: null argument");
    if (n < 0) return icm::fail(ICM_ERR_ARG, "icm_run_substeps_noalloc: negative substep count");
    if (p->GridX < 4 || p->GridY < 4) return icm::fail(ICM_ERR_ARG, "icm_run_substeps_noalloc: GridX/GridY below 4");
    const size_t nodes = (size_t)p->GridX * (size_t)p->GridY;
    if (nodes > kNoAllocMaxNodes)
        return icm::fail(ICM_ERR_ARG, "icm_run_substeps_noalloc: GridX*GridY = " + std::to_string(nodes) +
                                          " exceeds the fixed grid scratch of " + std::to_string(kNoAllocMaxNodes) +
                                          " nodes; use icm_run_substeps for larger grids");
    if (p->nPts < 0 || (p->nPts > 0 && p->nPtsPitch < (size_t)p->nPts))
        return icm::fail(ICM_ERR_ARG, "icm_run_substeps_noalloc: nPtsPitch smaller than nPts");
    if (p->n_indenter_subdivisions < 1) return icm::fail(ICM_ERR_ARG, "icm_run_substeps_noalloc: no force bins");
    if (!(p->cellsize > 0) || !(p->InitialTimeStep > 0) || p->UpdateEveryNthStep < 1)
        return icm::fail(ICM_ERR_ARG, "icm_run_substeps_noalloc: cellsize, time step or frame length not positive");
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    double *grid = nullptr;
    int rc = grid_address(s, &grid);
    if (rc) return rc;
    if (n == 0) return ICM_OK;

    icy_SimParams P = *p;
    P.grid_array = grid;
    P.nGridPitch = nodes;
    P.pts_array = pts;
    P.indenter_force_accumulator = bins;
    P.GridTotal = (int)nodes;
    const int tp = P.tpb_P2G > 0 ? P.tpb_P2G : 256, tu = P.tpb_Upd > 0 ? P.tpb_Upd : 512;
    const int tg = P.tpb_G2P > 0 ? P.tpb_G2P : 128;
    double t = p->SimulationTime;
    for (int k = 1; k <= n; k++) {
        t += P.InitialTimeStep;
        P.indenter_x = P.indenter_x_initial + t * P.IndVelocity;
        cudaError_t e = cudaMemsetAsync(grid, 0, sizeof(double) * 3 * nodes, s);
        if (e != cudaSuccess) return icm::fail(ICM_ERR_CUDA, std::string("grid clear: ") + cudaGetErrorString(e));
        if (P.nPts > 0) icm::k_p2g_ref64<<<(P.nPts + tp - 1) / tp, tp, 0, s>>>(P, err);
        icm::k_update_ref64<<<(int)((nodes + tu - 1) / tu), tu, 0, s>>>(P, P.indenter_x, P.indenter_y, nullptr);
        if (P.nPts > 0)
            icm::k_g2p_ref64<<<(P.nPts + tg - 1) / tg, tg, 0, s>>>(P, (p->SimulationStep + k) % P.UpdateEveryNthStep == 0);
        e = cudaGetLastError();
        if (e != cudaSuccess) return icm::fail(ICM_ERR_CUDA, std::string("substep launch: ") + cudaGetErrorString(e));
    }
    p->SimulationStep += n;
    p->SimulationTime = t;
    p->indenter_x = P.indenter_x;
    return ICM_OK;
}
