// mlp.cuh -- the learned Drucker-Prager projection: a 6 -> 64 -> 64 -> 3
// MLP (GELU, BF16 weights and activations, FP32 accumulation) standing in
// for Wolper_Drucker_Prager (gpu_implementation5.cu:48-94) in principal
// space.
//
// Features of a crushed particle, from the singular values s0 >= s1 of its
// trial elastic deformation gradient and Jp_inv:
//   x = [1e3 (s0 - 1), 1e3 (s1 - 1), 1e2 (Jp_inv - 1),
//        kappa * 1e-9, tan(phi), IceShearStrength * 1e-7]
// targets (what the exact projection changes):
//   y = [1e3 (s0' - s0), 1e3 (s1' - s1), 1e2 (Jp_inv' - Jp_inv)].
// The network sees (x - x_mu) / x_sd and predicts (y - y_mu) / y_sd.
//
// Parameters, FP32, in this order (kMlpFloats values): W1[64][6], b1[64],
// W2[64][64], b2[64], W3[3][64], b3[3], x_mu[6], x_sd[6], y_mu[3], y_sd[3].
// W[o][i] maps input i to output o.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>

#include "mpm_math64.cuh"

namespace icm {

constexpr int kMlpIn = 6, kMlpHid = 64, kMlpOut = 3;
constexpr int kOffW1 = 0, kOffB1 = kOffW1 + kMlpHid * kMlpIn, kOffW2 = kOffB1 + kMlpHid,
              kOffB2 = kOffW2 + kMlpHid * kMlpHid, kOffW3 = kOffB2 + kMlpHid, kOffB3 = kOffW3 + kMlpOut * kMlpHid,
              kOffXMu = kOffB3 + kMlpOut, kOffXSd = kOffXMu + kMlpIn, kOffYMu = kOffXSd + kMlpIn,
              kOffYSd = kOffYMu + kMlpOut, kMlpFloats = kOffYSd + kMlpOut;

// padded input width (K of the first layer) of the tensor-core forms
constexpr int kMlpInPad = 16;

__host__ __device__ __forceinline__ void mlp_features(const icy_SimParams &P, double s0, double s1, double jp,
                                                      float x[kMlpIn])
{
    x[0] = (float)(1e3 * (s0 - 1.0));
    x[1] = (float)(1e3 * (s1 - 1.0));
    x[2] = (float)(1e2 * (jp - 1.0));
    x[3] = (float)(P.kappa * 1e-9);
    x[4] = (float)P.DP_tan_phi;
    x[5] = (float)(P.IceShearStrength * 1e-7);
}

__host__ __device__ __forceinline__ void mlp_targets(double s0, double s1, double jp, double s0n, double s1n,
                                                     double jpn, float y[kMlpOut])
{
    y[0] = (float)(1e3 * (s0n - s0));
    y[1] = (float)(1e3 * (s1n - s1));
    y[2] = (float)(1e2 * (jpn - jp));
}

// tanh form of GELU and its derivative
__device__ __forceinline__ float gelu(float z)
{
    const float c = 0.7978845608028654f, a = 0.044715f;
    return 0.5f * z * (1.0f + tanhf(c * (z + a * z * z * z)));
}
__device__ __forceinline__ float gelu_grad(float z)
{
    const float c = 0.7978845608028654f, a = 0.044715f;
    const float th = tanhf(c * (z + a * z * z * z));
    return 0.5f * (1.0f + th) + 0.5f * z * (1.0f - th * th) * c * (1.0f + 3.0f * a * z * z);
}

// Weights of the warp form, BF16, [row = output][col = input] with inputs
// contiguous: W1 [64][16] (inputs padded with zeros), W2 [64][64], W3 [8][64]
// (outputs padded with zero rows), then FP32 b1[64], b2[64], b3[8] and the
// normalisation x_mu[8], 1/x_sd[8], y_mu[4], y_sd[4].
struct MlpWarpNet {
    __nv_bfloat16 W1[kMlpHid * kMlpInPad];
    __nv_bfloat16 W2[kMlpHid * kMlpHid];
    __nv_bfloat16 W3[8 * kMlpHid];
    float b1[kMlpHid], b2[kMlpHid], b3[8];
    float x_mu[8], x_isd[8], y_mu[4], y_sd[4];
};

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}

__device__ __forceinline__ uint32_t ldg_u32(const __nv_bfloat16 *p)
{
    return __ldg(reinterpret_cast<const unsigned int *>(p));
}

// GELU of the warp form, on the hardware tanh approximation (tanh.approx.f32,
// relative error about 2^-11, below the BF16 rounding the activation gets)
__device__ __forceinline__ float gelu_fast(float z)
{
    const float c = 0.7978845608028654f, a = 0.044715f;
    float th, u = c * (z + a * z * z * z);
    asm("tanh.approx.f32 %0, %1;" : "=f"(th) : "f"(u));
    return 0.5f * z * (1.0f + th);
}

// D += A B for one m16n8k16 tile (BF16 in, FP32 accumulate)
__device__ __forceinline__ void mma_bf16_16816(float d[4], const uint32_t a[4], uint32_t b0, uint32_t b1)
{
    asm volatile("mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                 "{%0,%1,%2,%3};"
                 : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
                 : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// One warp evaluates the network on 32 rows. row points at 32 rows of 16
// bytes: on entry row r holds the 8 BF16 normalised inputs of row r (the 6
// features, then zeros; inputs 8-15 of the K = 16 fragment are zero and not
// stored), on return its first 3 floats are the normalised outputs.
// Warp-collective: every lane of the warp calls it. A layer's accumulator
// tiles (two adjacent 8-column tiles) are the next layer's input fragment,
// so the activations stay in registers; weights are read through L1 from N.
static __device__ __noinline__ void warp_mlp(const MlpWarpNet *__restrict__ N, unsigned char *row)
{
    const __nv_bfloat16 *xrow = reinterpret_cast<const __nv_bfloat16 *>(row);
    float *yrow = reinterpret_cast<float *>(row);
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    __syncwarp();
#pragma unroll 1
    for (int mt = 0; mt < 2; mt++) {
        const int r0 = mt * 16 + g, r1 = r0 + 8;
        uint32_t a1[4];
        a1[0] = *reinterpret_cast<const uint32_t *>(xrow + r0 * 8 + 2 * t);
        a1[1] = *reinterpret_cast<const uint32_t *>(xrow + r1 * 8 + 2 * t);
        a1[2] = 0u;
        a1[3] = 0u;
        // layer 1 -> layer-2 input fragments (4 K-tiles of 16 hidden units)
        uint32_t a2[4][4];
#pragma unroll
        for (int kt = 0; kt < 4; kt++) {
            float c[2][4];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int nt = 2 * kt + h, n = nt * 8 + g;
                const float bb0 = N->b1[nt * 8 + 2 * t], bb1 = N->b1[nt * 8 + 2 * t + 1];
                c[h][0] = bb0; c[h][1] = bb1; c[h][2] = bb0; c[h][3] = bb1;
                mma_bf16_16816(c[h], a1, ldg_u32(N->W1 + n * 16 + 2 * t), ldg_u32(N->W1 + n * 16 + 2 * t + 8));
            }
            a2[kt][0] = pack_bf16(gelu_fast(c[0][0]), gelu_fast(c[0][1]));
            a2[kt][1] = pack_bf16(gelu_fast(c[0][2]), gelu_fast(c[0][3]));
            a2[kt][2] = pack_bf16(gelu_fast(c[1][0]), gelu_fast(c[1][1]));
            a2[kt][3] = pack_bf16(gelu_fast(c[1][2]), gelu_fast(c[1][3]));
        }
        // layer 2, 16 hidden units at a time, streamed into layer 3
        float c3[4];
        {
            const float bb0 = N->b3[2 * t], bb1 = N->b3[2 * t + 1];
            c3[0] = bb0; c3[1] = bb1; c3[2] = bb0; c3[3] = bb1;
        }
#pragma unroll 1
        for (int k3 = 0; k3 < 4; k3++) {
            float c[2][4];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int nt = 2 * k3 + h, n = nt * 8 + g;
                const float bb0 = N->b2[nt * 8 + 2 * t], bb1 = N->b2[nt * 8 + 2 * t + 1];
                c[h][0] = bb0; c[h][1] = bb1; c[h][2] = bb0; c[h][3] = bb1;
#pragma unroll
                for (int kt = 0; kt < 4; kt++)
                    mma_bf16_16816(c[h], a2[kt], ldg_u32(N->W2 + n * 64 + 16 * kt + 2 * t),
                                   ldg_u32(N->W2 + n * 64 + 16 * kt + 2 * t + 8));
            }
            uint32_t a3[4];
            a3[0] = pack_bf16(gelu_fast(c[0][0]), gelu_fast(c[0][1]));
            a3[1] = pack_bf16(gelu_fast(c[0][2]), gelu_fast(c[0][3]));
            a3[2] = pack_bf16(gelu_fast(c[1][0]), gelu_fast(c[1][1]));
            a3[3] = pack_bf16(gelu_fast(c[1][2]), gelu_fast(c[1][3]));
            mma_bf16_16816(c3, a3, ldg_u32(N->W3 + g * 64 + 16 * k3 + 2 * t),
                           ldg_u32(N->W3 + g * 64 + 16 * k3 + 2 * t + 8));
        }
        __syncwarp();  // every lane has read its inputs of this tile
        if (t < 2) {  // outputs 2t, 2t+1 (only 0..2 are real), over the inputs
            yrow[r0 * 4 + 2 * t] = c3[0];
            yrow[r0 * 4 + 2 * t + 1] = c3[1];
            yrow[r1 * 4 + 2 * t] = c3[2];
            yrow[r1 * 4 + 2 * t + 1] = c3[3];
        }
    }
    __syncwarp();
}

}  // namespace icm
