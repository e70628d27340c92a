// mlp.cu -- training and inference of the learned Drucker-Prager projection
// (mlp.cuh) on the tensor cores.
//
// Training: one CTA of 128 threads takes 128 samples (one row per thread,
// TMEM lane = row) through
//   forward   Z1 = X W1^T, H1 = gelu(Z1 + b1); Z2 = H1 W2^T, H2 = gelu(..);
//             Y = H2 W3^T + b3
//   backward  dZ3 = 2 (Y - T) / (3 B); dH2 = dZ3 W3; dZ2 = dH2 gelu'(..);
//             dH1 = dZ2 W2; dZ1 = dH1 gelu'(..)
//   weights   dW3^T = H2^T dZ3, dW2 = dZ2^T H1, dW1 = dZ1^T X
// with every product a tcgen05 BF16 MMA (M = 128 over samples, M = 64 over
// hidden units for the weight gradients) accumulating in TMEM; the per-CTA
// weight gradients go to an FP32 gradient buffer with atomics, and an Adam
// step (FP32 master weights) follows each batch.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "../../include/icempm.h"
#include "errors.h"
#include "mlp.cuh"
#include "tc05.cuh"

namespace icm {

namespace {

// BF16 operand tiles of the tensor-core form, K-major core-matrix layout
// (tc05.cuh): W1k [64 x 16], W2k [64 x 64], W3k [16 x 64] (rows >= 3 zero),
// W3Tk [64 x 16] (cols >= 3 zero), W2Tk [64 x 64].
struct MlpTcNet {
    __nv_bfloat16 W1k[64 * 16], W2k[64 * 64], W3k[16 * 64], W3Tk[64 * 16], W2Tk[64 * 64];
};

constexpr int kRows = 128;
// TMEM columns of the accumulators (32-aligned starts). Accumulators share
// columns where one is dead before the next is written: Z3 is read before
// dH2 is formed, Z2 (read for gelu' in dH2's epilogue) before dH1, dH2
// (read in that epilogue) before dW2, dW3^T before dW1; Z1 stays for
// gelu' of the last step. 256 columns let two CTAs share an SM's 512.
constexpr uint32_t kTmemCols = 256;
constexpr int cZ1 = 0, cZ2 = 64, cDH1 = 64, cZ3 = 128, cDH2 = 128, cDW2 = 128, cDW3T = 192, cDW1 = 192;
constexpr int kWaitPolls = 1 << 24;

// shared-memory layout of k_mlp_tile (bytes). dZ3 takes X's tile (read
// only by the first product) and dZ2^T takes H2^T's (last read by the
// product for dW3^T, which completes before dZ2 is formed): 98 KB, two CTAs
// per SM.
constexpr int sW1 = 0, sW2 = sW1 + 2048, sW3 = sW2 + 8192, sW3T = sW3 + 2048, sW2T = sW3T + 2048,
              sX = sW2T + 8192, sXT = sX + 4096, sH1 = sXT + 4096, sH1T = sH1 + 16384, sH2 = sH1T + 16384,
              sH2T = sH2 + 16384, sDZ3T = sH2T + 16384, kTileSmem = sDZ3T + 4096;
constexpr int sDZ3 = sX, sDZ2T = sH2T;

__device__ __forceinline__ void put_bf16(unsigned char *base, int row, int k, int K, float v)
{
    *reinterpret_cast<__nv_bfloat16 *>(base + tc05::kmajor_offset(row, k, K)) = __float2bfloat16(v);
}

__device__ __forceinline__ uint32_t sample_index(uint32_t seed, int step, int row, int n)
{
    uint32_t h = seed ^ ((uint32_t)step * 0x9E3779B9u) ^ ((uint32_t)row * 0x85EBCA6Bu);
    h ^= h >> 16;
    h *= 0x7feb352du;
    h ^= h >> 15;
    h *= 0x846ca68bu;
    h ^= h >> 16;
    return h % (uint32_t)n;
}

__device__ __forceinline__ float warp_sum(float v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

struct TileArgs {
    const float *X, *Y;      // raw features [n][6], targets [n][3]
    int n;
    int sequential;          // rows blockIdx*128 + r (else hashed samples)
    uint32_t seed;
    int step;
    float inv_count;         // 1 / (3 * samples in the batch)
    const MlpTcNet *tc;      // BF16 operand tiles
    const float *net;        // FP32 parameters (biases, normalisation)
    float *grad;             // FP32 gradient (same layout as net), accumulated
    size_t grad_stride;      // CTA b adds into grad + b * grad_stride (0: all into one)
    float *loss;             // accumulated mean squared error
    float *Yout;             // inference: denormalised outputs [n][3]
    int *status;             // set to 1 when a wait gives up
};

template <bool TRAIN>
__global__ void __launch_bounds__(kRows) k_mlp_tile(const TileArgs a)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ __align__(8) uint64_t mbar;
    __shared__ uint32_t s_tmem;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const float *net = a.net;
    // this CTA's gradient: its own slice in training, so that the CTAs of a
    // step do not contend for the same addresses (the Adam step adds the
    // slices up)
    float *grad = a.grad + (size_t)blockIdx.x * a.grad_stride;

    // sample of this row
    int idx;
    bool valid;
    if (a.sequential) {
        idx = blockIdx.x * kRows + tid;
        valid = idx < a.n;
    } else {
        idx = (int)sample_index(a.seed, a.step, blockIdx.x * kRows + tid, a.n);
        valid = true;
    }
    // operand tiles of the weights
    {
        const uint4 *src = reinterpret_cast<const uint4 *>(a.tc);
        uint4 *dst = reinterpret_cast<uint4 *>(sm + sW1);
        const int nvec = (int)(sizeof(MlpTcNet) / 16);
        for (int i = tid; i < nvec; i += kRows) dst[i] = src[i];
    }
    // normalised inputs: row tid of X, column tid of X^T
#pragma unroll
    for (int k = 0; k < kMlpInPad; k++) {
        float v = 0.f;
        if (k < kMlpIn && valid) v = (a.X[(size_t)idx * kMlpIn + k] - net[kOffXMu + k]) / net[kOffXSd + k];
        put_bf16(sm + sX, tid, k, 16, v);
        if (TRAIN) put_bf16(sm + sXT, k, tid, kRows, v);
    }
    if (tid == 0) tc05::mbar_init(&mbar, 1);
    if (warp == 0) tc05::alloc(&s_tmem, kTmemCols);
    tc05::fence_smem_for_mma();
    tc05::fence_before_sync();
    __syncthreads();
    tc05::fence_after_sync();
    const uint32_t tmem = s_tmem;
    uint32_t phase = 0;
    bool ok = true;
    auto wait_mma = [&]() {
        ok = tc05::mbar_wait(&mbar, phase, kWaitPolls) && ok;
        phase ^= 1;
        tc05::fence_after_sync();
    };
    auto publish = [&]() {  // shared-memory operands written by all threads -> MMA
        tc05::fence_smem_for_mma();
        tc05::fence_before_sync();
        __syncthreads();
        tc05::fence_after_sync();
    };
    const uint32_t id128x64 = tc05::idesc_bf16(128, 64), id128x16 = tc05::idesc_bf16(128, 16);
    const uint32_t id64x16 = tc05::idesc_bf16(64, 16), id64x64 = tc05::idesc_bf16(64, 64);

    // ---- Z1 = X W1^T
    if (tid == 0) {
        tc05::mma(tmem + cZ1, tc05::desc_kmajor(sm + sX, 16), tc05::desc_kmajor(sm + sW1, 16), id128x64, false);
        tc05::commit(&mbar);
    }
    wait_mma();
    float z[16];
#pragma unroll 1
    for (int c0 = 0; c0 < 64; c0 += 16) {
        tc05::ld16(tc05::taddr(tmem, warp, cZ1 + c0), z);
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const float h = gelu(z[j] + net[kOffB1 + c0 + j]);
            put_bf16(sm + sH1, tid, c0 + j, 64, h);
            if (TRAIN) put_bf16(sm + sH1T, c0 + j, tid, kRows, h);
        }
    }
    publish();
    // ---- Z2 = H1 W2^T
    if (tid == 0) {
        for (int kk = 0; kk < 4; kk++)
            tc05::mma(tmem + cZ2, tc05::desc_kmajor(sm + sH1 + 256 * kk, 64), tc05::desc_kmajor(sm + sW2 + 256 * kk, 64),
                      id128x64, kk > 0);
        tc05::commit(&mbar);
    }
    wait_mma();
#pragma unroll 1
    for (int c0 = 0; c0 < 64; c0 += 16) {
        tc05::ld16(tc05::taddr(tmem, warp, cZ2 + c0), z);
#pragma unroll
        for (int j = 0; j < 16; j++) {
            const float h = gelu(z[j] + net[kOffB2 + c0 + j]);
            put_bf16(sm + sH2, tid, c0 + j, 64, h);
            if (TRAIN) put_bf16(sm + sH2T, c0 + j, tid, kRows, h);
        }
    }
    publish();
    // ---- Y = H2 W3^T + b3
    if (tid == 0) {
        for (int kk = 0; kk < 4; kk++)
            tc05::mma(tmem + cZ3, tc05::desc_kmajor(sm + sH2 + 256 * kk, 64), tc05::desc_kmajor(sm + sW3 + 256 * kk, 64),
                      id128x16, kk > 0);
        tc05::commit(&mbar);
    }
    wait_mma();
    tc05::ld16(tc05::taddr(tmem, warp, cZ3), z);
    float y[kMlpOut];
#pragma unroll
    for (int o = 0; o < kMlpOut; o++) y[o] = z[o] + net[kOffB3 + o];

    if (!TRAIN) {
        if (valid)
            for (int o = 0; o < kMlpOut; o++)
                a.Yout[(size_t)idx * kMlpOut + o] = y[o] * net[kOffYSd + o] + net[kOffYMu + o];
    } else {
        // ---- loss and dZ3
        float dy[kMlpOut], se = 0.f;
#pragma unroll
        for (int o = 0; o < kMlpOut; o++) {
            const float t = valid ? (a.Y[(size_t)idx * kMlpOut + o] - net[kOffYMu + o]) / net[kOffYSd + o] : y[o];
            const float d = y[o] - t;
            se += d * d;
            dy[o] = valid ? 2.f * d * a.inv_count : 0.f;
        }
#pragma unroll
        for (int o = 0; o < 16; o++) {
            const float v = o < kMlpOut ? dy[o] : 0.f;
            put_bf16(sm + sDZ3, tid, o, 16, v);
            put_bf16(sm + sDZ3T, o, tid, kRows, v);
        }
        se = warp_sum(se);
        if (lane == 0) atomicAdd(a.loss, se * a.inv_count);
#pragma unroll
        for (int o = 0; o < kMlpOut; o++) {
            const float s = warp_sum(dy[o]);
            if (lane == 0) atomicAdd(&grad[kOffB3 + o], s);
        }
        publish();
        // ---- dH2 = dZ3 W3 ; dW3^T = H2^T dZ3
        if (tid == 0) {
            tc05::mma(tmem + cDH2, tc05::desc_kmajor(sm + sDZ3, 16), tc05::desc_kmajor(sm + sW3T, 16), id128x64, false);
            for (int kk = 0; kk < 8; kk++)
                tc05::mma(tmem + cDW3T, tc05::desc_kmajor(sm + sH2T + 256 * kk, kRows),
                          tc05::desc_kmajor(sm + sDZ3T + 256 * kk, kRows), id64x16, kk > 0);
            tc05::commit(&mbar);
        }
        wait_mma();
        float dh[16];
#pragma unroll 1
        for (int c0 = 0; c0 < 64; c0 += 16) {
            tc05::ld16(tc05::taddr(tmem, warp, cDH2 + c0), dh);
            tc05::ld16(tc05::taddr(tmem, warp, cZ2 + c0), z);
#pragma unroll
            for (int j = 0; j < 16; j++) {
                const float d = dh[j] * gelu_grad(z[j] + net[kOffB2 + c0 + j]);
                put_bf16(sm + sH2, tid, c0 + j, 64, d);  // dZ2 over H2 (no longer read)
                put_bf16(sm + sDZ2T, c0 + j, tid, kRows, d);
                const float s = warp_sum(d);
                if (lane == 0) atomicAdd(&grad[kOffB2 + c0 + j], s);
            }
        }
        // dW3^T rows (hidden unit 16 warp + lane for lanes < 16)
        tc05::ld16(tc05::taddr(tmem, warp, cDW3T), dh);
        if (lane < 16)
            for (int o = 0; o < kMlpOut; o++) atomicAdd(&grad[kOffW3 + o * kMlpHid + warp * 16 + lane], dh[o]);
        publish();
        // ---- dH1 = dZ2 W2 ; dW2 = dZ2^T H1
        if (tid == 0) {
            for (int kk = 0; kk < 4; kk++)
                tc05::mma(tmem + cDH1, tc05::desc_kmajor(sm + sH2 + 256 * kk, 64),
                          tc05::desc_kmajor(sm + sW2T + 256 * kk, 64), id128x64, kk > 0);
            for (int kk = 0; kk < 8; kk++)
                tc05::mma(tmem + cDW2, tc05::desc_kmajor(sm + sDZ2T + 256 * kk, kRows),
                          tc05::desc_kmajor(sm + sH1T + 256 * kk, kRows), id64x64, kk > 0);
            tc05::commit(&mbar);
        }
        wait_mma();
#pragma unroll 1
        for (int c0 = 0; c0 < 64; c0 += 16) {
            tc05::ld16(tc05::taddr(tmem, warp, cDH1 + c0), dh);
            tc05::ld16(tc05::taddr(tmem, warp, cZ1 + c0), z);
#pragma unroll
            for (int j = 0; j < 16; j++) {
                const float d = dh[j] * gelu_grad(z[j] + net[kOffB1 + c0 + j]);
                put_bf16(sm + sH1, c0 + j, tid, kRows, d);  // dZ1^T over H1 (no longer read)
                const float s = warp_sum(d);
                if (lane == 0) atomicAdd(&grad[kOffB1 + c0 + j], s);
            }
        }
#pragma unroll 1
        for (int c0 = 0; c0 < 64; c0 += 16) {
            tc05::ld16(tc05::taddr(tmem, warp, cDW2 + c0), dh);
            if (lane < 16)
                for (int j = 0; j < 16; j++) atomicAdd(&grad[kOffW2 + (warp * 16 + lane) * kMlpHid + c0 + j], dh[j]);
        }
        publish();
        // ---- dW1 = dZ1^T X
        if (tid == 0) {
            for (int kk = 0; kk < 8; kk++)
                tc05::mma(tmem + cDW1, tc05::desc_kmajor(sm + sH1 + 256 * kk, kRows),
                          tc05::desc_kmajor(sm + sXT + 256 * kk, kRows), id64x16, kk > 0);
            tc05::commit(&mbar);
        }
        wait_mma();
        tc05::ld16(tc05::taddr(tmem, warp, cDW1), dh);
        if (lane < 16)
            for (int i = 0; i < kMlpIn; i++) atomicAdd(&grad[kOffW1 + (warp * 16 + lane) * kMlpIn + i], dh[i]);
    }
    if (!ok && a.status) atomicExch(a.status, 1);
    tc05::fence_before_sync();
    __syncthreads();
    tc05::fence_after_sync();
    if (warp == 0) tc05::dealloc(tmem, kTmemCols);
}

// FP32 parameters -> the BF16 operand tiles of both tensor-core forms
__global__ void k_mlp_prep(const float *net, MlpTcNet *tc, MlpWarpNet *wn)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    auto put = [](__nv_bfloat16 *tile, int row, int k, int K, float w) {
        *reinterpret_cast<__nv_bfloat16 *>(reinterpret_cast<unsigned char *>(tile) + tc05::kmajor_offset(row, k, K)) =
            __float2bfloat16(w);
    };
    if (i < 64 * 16) {  // W1 [64][16]
        const int o = i / 16, k = i % 16;
        const float w = k < kMlpIn ? net[kOffW1 + o * kMlpIn + k] : 0.f;
        put(tc->W1k, o, k, 16, w);
        if (wn) wn->W1[o * 16 + k] = __float2bfloat16(w);
    }
    if (i < 64 * 64) {  // W2 [64][64] and its transpose
        const int o = i / 64, k = i % 64;
        const float w = net[kOffW2 + o * 64 + k];
        put(tc->W2k, o, k, 64, w);
        put(tc->W2Tk, k, o, 64, w);
        if (wn) wn->W2[o * 64 + k] = __float2bfloat16(w);
    }
    if (i < 16 * 64) {  // W3 [16][64] (3 real rows) and its transpose [64][16]
        const int o = i / 64, k = i % 64;
        const float w = o < kMlpOut ? net[kOffW3 + o * 64 + k] : 0.f;
        put(tc->W3k, o, k, 64, w);
        put(tc->W3Tk, k, o, 16, w);
        if (wn && o < 8) wn->W3[o * 64 + k] = __float2bfloat16(w);
    }
    if (wn && i < 64) {
        wn->b1[i] = net[kOffB1 + i];
        wn->b2[i] = net[kOffB2 + i];
        if (i < 8) {
            wn->b3[i] = i < kMlpOut ? net[kOffB3 + i] : 0.f;
            wn->x_mu[i] = i < kMlpIn ? net[kOffXMu + i] : 0.f;
            wn->x_isd[i] = i < kMlpIn ? 1.0f / net[kOffXSd + i] : 0.f;
        }
        if (i < 4) {
            wn->y_mu[i] = i < kMlpOut ? net[kOffYMu + i] : 0.f;
            wn->y_sd[i] = i < kMlpOut ? net[kOffYSd + i] : 0.f;
        }
    }
}

// Adam on the weights and biases (not the normalisation)
// Adam step on the sum of nslices gradient slices (stride floats apart)
__global__ void k_mlp_adam(float *net, float *m, float *v, const float *grad, int nslices, size_t stride, int count,
                           float lr, float b1, float b2, float eps, float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    float g = 0.f;
    for (int b = 0; b < nslices; b++) g += grad[(size_t)b * stride + i];
    const float mi = b1 * m[i] + (1.f - b1) * g, vi = b2 * v[i] + (1.f - b2) * g * g;
    m[i] = mi;
    v[i] = vi;
    net[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
}

// the warp form over a batch (tests and measurements of the in-kernel form)
__global__ void __launch_bounds__(128) k_mlp_warp_infer(const MlpWarpNet *N, const float *X, int n, float *Yout)
{
    __shared__ __align__(16) unsigned char rows[4][32 * 16];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r = (blockIdx.x * 4 + warp) * 32 + lane;
    __nv_bfloat16 *xrow = reinterpret_cast<__nv_bfloat16 *>(rows[warp]);
#pragma unroll
    for (int k = 0; k < 8; k++) {
        float v = 0.f;
        if (k < kMlpIn && r < n) v = (X[(size_t)r * kMlpIn + k] - N->x_mu[k]) * N->x_isd[k];
        xrow[lane * 8 + k] = __float2bfloat16(v);
    }
    warp_mlp(N, rows[warp]);
    const float *yrow = reinterpret_cast<const float *>(rows[warp]);
    if (r < n)
        for (int o = 0; o < kMlpOut; o++) Yout[(size_t)r * kMlpOut + o] = yrow[lane * 4 + o] * N->y_sd[o] + N->y_mu[o];
}

// harvested trial states (H00, H01, H10, H11, Jp_inv, meta word) ->
// features and exact targets
__global__ void k_mlp_label(const icy_SimParams P, const float *harvest, int n, float *X, float *Y)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float *h = harvest + (size_t)i * 6;
    const M2d F = {1.0 + (double)h[0], (double)h[1], (double)h[2], 1.0 + (double)h[3]};
    const double jp = h[4];
    const Svd64 d = svd2x2_64(F);
    float x[kMlpIn], y[kMlpOut];
    mlp_features(P, d.s0, d.s1, jp, x);
    const DpResult r = dp_project64(P, d.s0, d.s1, jp);
    mlp_targets(d.s0, d.s1, jp, r.s0, r.s1, r.jp, y);
    for (int k = 0; k < kMlpIn; k++) X[(size_t)i * kMlpIn + k] = x[k];
    for (int k = 0; k < kMlpOut; k++) Y[(size_t)i * kMlpOut + k] = y[k];
}

// ------------------------------------------------------------ host side

template <class T> struct DevBuf {
    T *p = nullptr;
    ~DevBuf()
    {
        if (p) cudaFree(p);
    }
    int alloc(size_t n)
    {
        return cudaMalloc((void **)&p, sizeof(T) * std::max<size_t>(n, 1)) == cudaSuccess
                   ? ICM_OK
                   : icm::fail(ICM_ERR_NOMEM, "mlp: device allocation failed");
    }
};

// the opt-in is per device (cudaFuncSetAttribute acts on the current one)
int set_tile_smem()
{
    constexpr int kMaxDevices = 64;
    static bool done[kMaxDevices] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return icm::fail(ICM_ERR_CUDA, "mlp: cudaGetDevice");
    if (dev >= 0 && dev < kMaxDevices && done[dev]) return ICM_OK;
    if (cudaFuncSetAttribute(k_mlp_tile<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmem) != cudaSuccess ||
        cudaFuncSetAttribute(k_mlp_tile<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmem) != cudaSuccess)
        return icm::fail(ICM_ERR_CUDA, "mlp: shared-memory opt-in failed");
    if (dev >= 0 && dev < kMaxDevices) done[dev] = true;
    return ICM_OK;
}

int finish_device(const char *what, const int *d_status)
{
    if (cudaDeviceSynchronize() != cudaSuccess)
        return icm::fail(ICM_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(cudaGetLastError()));
    int s = 0;
    if (d_status && cudaMemcpy(&s, d_status, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess)
        return icm::fail(ICM_ERR_CUDA, std::string(what) + ": status copy");
    if (s) return icm::fail(ICM_ERR_CUDA, std::string(what) + ": a tensor-core wait gave up");
    return ICM_OK;
}

int select_device(int device)
{
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        return icm::fail(ICM_ERR_NODEVICE, "No avaialble CUDA devices");
    if (device < 0 || device >= count) return icm::fail(ICM_ERR_ARG, "mlp: device index out of range");
    if (cudaSetDevice(device) != cudaSuccess) return icm::fail(ICM_ERR_CUDA, "mlp: cudaSetDevice");
    return ICM_OK;
}

void launch_prep(const float *net, MlpTcNet *tc, MlpWarpNet *wn, cudaStream_t s = 0)
{
    k_mlp_prep<<<(64 * 64 + 255) / 256, 256, 0, s>>>(net, tc, wn);
}

}  // namespace

// used by the surrogate form of the substep (device_layer.cu)
int mlp_prepare_warp_net(const float *host_net, MlpWarpNet **out)
{
    DevBuf<float> net;
    DevBuf<MlpTcNet> tc;
    int rc;
    if ((rc = net.alloc(kMlpFloats)) || (rc = tc.alloc(1))) return rc;
    MlpWarpNet *wn = nullptr;
    if (cudaMalloc((void **)&wn, sizeof(MlpWarpNet)) != cudaSuccess) return icm::fail(ICM_ERR_NOMEM, "mlp: allocation");
    cudaMemcpy(net.p, host_net, sizeof(float) * kMlpFloats, cudaMemcpyHostToDevice);
    launch_prep(net.p, tc.p, wn);
    if ((rc = finish_device("mlp prep", nullptr))) {
        cudaFree(wn);
        return rc;
    }
    *out = wn;
    return ICM_OK;
}

int mlp_label(const icy_SimParams &P, const float *d_harvest, int n, float *d_x, float *d_y, cudaStream_t s)
{
    if (n <= 0) return ICM_OK;
    k_mlp_label<<<(n + 127) / 128, 128, 0, s>>>(P, d_harvest, n, d_x, d_y);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return icm::fail(ICM_ERR_CUDA, std::string("k_mlp_label: ") + cudaGetErrorString(e));
    return ICM_OK;
}

}  // namespace icm

using namespace icm;

extern "C" int icm_mlp_floats(void) { return kMlpFloats; }

extern "C" int icm_mlp_normalise(float *net, const float *x, const float *y, int n)
{
    if (!net || !x || !y || n < 2) return icm::fail(ICM_ERR_ARG, "icm_mlp_normalise: bad arguments");
    auto stats = [&](const float *a, int dim, int k, float &mu, float &sd) {
        double s = 0, q = 0;
        for (int i = 0; i < n; i++) s += a[(size_t)i * dim + k];
        const double m = s / n;
        for (int i = 0; i < n; i++) {
            const double d = a[(size_t)i * dim + k] - m;
            q += d * d;
        }
        const double v = std::sqrt(q / (n - 1));
        mu = (float)m;
        sd = (float)(v > 1e-6 * std::max(1.0, std::fabs(m)) ? v : 1.0);
    };
    for (int k = 0; k < kMlpIn; k++) stats(x, kMlpIn, k, net[kOffXMu + k], net[kOffXSd + k]);
    for (int k = 0; k < kMlpOut; k++) stats(y, kMlpOut, k, net[kOffYMu + k], net[kOffYSd + k]);
    return ICM_OK;
}

extern "C" int icm_mlp_train(int device, const float *x, const float *y, int n, const icm_mlp_train_cfg *cfg,
                             float *net_io, float *loss_hist)
{
    if (!x || !y || !cfg || !net_io || n < 1 || cfg->steps < 0 || cfg->batch_tiles < 1)
        return icm::fail(ICM_ERR_ARG, "icm_mlp_train: bad arguments");
    int rc = select_device(device);
    if (rc || (rc = set_tile_smem())) return rc;
    DevBuf<float> X, Y, net, m, v, grad, loss;
    DevBuf<MlpTcNet> tc;
    DevBuf<int> status;
    const int steps = cfg->steps;
    if ((rc = X.alloc((size_t)n * kMlpIn)) || (rc = Y.alloc((size_t)n * kMlpOut)) || (rc = net.alloc(kMlpFloats)) ||
        (rc = m.alloc(kMlpFloats)) || (rc = v.alloc(kMlpFloats)) ||
        (rc = grad.alloc((size_t)std::max(cfg->batch_tiles, 1) * kMlpFloats)) ||
        (rc = loss.alloc(std::max(steps, 1))) || (rc = tc.alloc(1)) || (rc = status.alloc(1)))
        return rc;
    cudaMemcpy(X.p, x, sizeof(float) * n * kMlpIn, cudaMemcpyHostToDevice);
    cudaMemcpy(Y.p, y, sizeof(float) * n * kMlpOut, cudaMemcpyHostToDevice);
    cudaMemcpy(net.p, net_io, sizeof(float) * kMlpFloats, cudaMemcpyHostToDevice);
    cudaMemset(m.p, 0, sizeof(float) * kMlpFloats);
    cudaMemset(v.p, 0, sizeof(float) * kMlpFloats);
    cudaMemset(loss.p, 0, sizeof(float) * std::max(steps, 1));
    cudaMemset(status.p, 0, sizeof(int));
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    TileArgs a{};
    a.X = X.p;
    a.Y = Y.p;
    a.n = n;
    a.sequential = 0;
    a.seed = cfg->seed;
    a.inv_count = 1.0f / (3.0f * kRows * cfg->batch_tiles);
    a.tc = tc.p;
    a.net = net.p;
    a.grad = grad.p;
    a.grad_stride = kMlpFloats;
    a.status = status.p;
    const int nw = kOffXMu;  // weights and biases
    for (int s = 0; s < steps; s++) {
        launch_prep(net.p, tc.p, nullptr);
        cudaMemsetAsync(grad.p, 0, sizeof(float) * kMlpFloats * (size_t)cfg->batch_tiles);
        a.step = s;
        a.loss = loss.p + s;
        k_mlp_tile<true><<<cfg->batch_tiles, kRows, kTileSmem>>>(a);
        // cosine decay from lr to lr/20
        const float frac = steps > 1 ? (float)s / (float)(steps - 1) : 0.f;
        const float lr = cfg->lr * (0.05f + 0.95f * 0.5f * (1.0f + std::cos(3.14159265f * frac)));
        const float c1 = 1.0f / (1.0f - std::pow(b1, (float)(s + 1))), c2 = 1.0f / (1.0f - std::pow(b2, (float)(s + 1)));
        k_mlp_adam<<<(nw + 255) / 256, 256>>>(net.p, m.p, v.p, grad.p, cfg->batch_tiles, kMlpFloats, nw, lr, b1, b2,
                                              eps, c1, c2);
    }
    if ((rc = finish_device("icm_mlp_train", status.p))) return rc;
    cudaMemcpy(net_io, net.p, sizeof(float) * kMlpFloats, cudaMemcpyDeviceToHost);
    if (loss_hist && steps > 0) cudaMemcpy(loss_hist, loss.p, sizeof(float) * steps, cudaMemcpyDeviceToHost);
    return ICM_OK;
}

extern "C" int icm_mlp_gradient(int device, const float *net_in, const float *x, const float *y, int n,
                                float *grad_out, float *loss_out)
{
    if (!net_in || !x || !y || !grad_out || n < 1) return icm::fail(ICM_ERR_ARG, "icm_mlp_gradient: bad arguments");
    int rc = select_device(device);
    if (rc || (rc = set_tile_smem())) return rc;
    DevBuf<float> X, Y, net, grad, loss;
    DevBuf<MlpTcNet> tc;
    DevBuf<int> status;
    if ((rc = X.alloc((size_t)n * kMlpIn)) || (rc = Y.alloc((size_t)n * kMlpOut)) || (rc = net.alloc(kMlpFloats)) ||
        (rc = grad.alloc(kMlpFloats)) || (rc = loss.alloc(1)) || (rc = tc.alloc(1)) || (rc = status.alloc(1)))
        return rc;
    cudaMemcpy(X.p, x, sizeof(float) * n * kMlpIn, cudaMemcpyHostToDevice);
    cudaMemcpy(Y.p, y, sizeof(float) * n * kMlpOut, cudaMemcpyHostToDevice);
    cudaMemcpy(net.p, net_in, sizeof(float) * kMlpFloats, cudaMemcpyHostToDevice);
    cudaMemset(grad.p, 0, sizeof(float) * kMlpFloats);
    cudaMemset(loss.p, 0, sizeof(float));
    cudaMemset(status.p, 0, sizeof(int));
    launch_prep(net.p, tc.p, nullptr);
    TileArgs a{};
    a.X = X.p;
    a.Y = Y.p;
    a.n = n;
    a.sequential = 1;
    a.inv_count = 1.0f / (3.0f * n);
    a.tc = tc.p;
    a.net = net.p;
    a.grad = grad.p;
    a.loss = loss.p;
    a.status = status.p;
    k_mlp_tile<true><<<(n + kRows - 1) / kRows, kRows, kTileSmem>>>(a);
    if ((rc = finish_device("icm_mlp_gradient", status.p))) return rc;
    cudaMemcpy(grad_out, grad.p, sizeof(float) * kMlpFloats, cudaMemcpyDeviceToHost);
    if (loss_out) cudaMemcpy(loss_out, loss.p, sizeof(float), cudaMemcpyDeviceToHost);
    return ICM_OK;
}

extern "C" int icm_mlp_infer(int device, const float *net_in, const float *x, int n, float *y_out, int warp_form)
{
    if (!net_in || !x || !y_out || n < 1) return icm::fail(ICM_ERR_ARG, "icm_mlp_infer: bad arguments");
    int rc = select_device(device);
    if (rc || (rc = set_tile_smem())) return rc;
    DevBuf<float> X, Yo, net;
    DevBuf<MlpTcNet> tc;
    DevBuf<MlpWarpNet> wn;
    DevBuf<int> status;
    if ((rc = X.alloc((size_t)n * kMlpIn)) || (rc = Yo.alloc((size_t)n * kMlpOut)) || (rc = net.alloc(kMlpFloats)) ||
        (rc = tc.alloc(1)) || (rc = wn.alloc(1)) || (rc = status.alloc(1)))
        return rc;
    cudaMemcpy(X.p, x, sizeof(float) * n * kMlpIn, cudaMemcpyHostToDevice);
    cudaMemcpy(net.p, net_in, sizeof(float) * kMlpFloats, cudaMemcpyHostToDevice);
    cudaMemset(status.p, 0, sizeof(int));
    launch_prep(net.p, tc.p, wn.p);
    if (warp_form) {
        k_mlp_warp_infer<<<(n + 127) / 128, 128>>>(wn.p, X.p, n, Yo.p);
    } else {
        TileArgs a{};
        a.X = X.p;
        a.n = n;
        a.sequential = 1;
        a.tc = tc.p;
        a.net = net.p;
        a.Yout = Yo.p;
        a.status = status.p;
        k_mlp_tile<false><<<(n + kRows - 1) / kRows, kRows, kTileSmem>>>(a);
    }
    if ((rc = finish_device("icm_mlp_infer", status.p))) return rc;
    cudaMemcpy(y_out, Yo.p, sizeof(float) * n * kMlpOut, cudaMemcpyDeviceToHost);
    return ICM_OK;
}
