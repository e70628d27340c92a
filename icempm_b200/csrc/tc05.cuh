// tc05.cuh -- thin wrappers over the sm_100a tensor-core instructions
// (tcgen05.*) and the mbarrier used to wait for them, for one-CTA
// (cta_group::1) BF16 x BF16 -> FP32 MMAs with both operands in shared
// memory.
//
// Operands are K-major without swizzle: the tile is stored as 8-row x
// 16-byte "core matrices"; element (row, k) of a tile with K columns sits at
// byte ((row/8) * (K/8) + k/8) * 128 + (row%8) * 16 + (k%8) * 2, so the
// descriptor's leading-byte offset (next 8 columns of K) is 128 and its
// stride-byte offset (next 8 rows) is (K/8) * 128. One MMA consumes K = 16;
// the next 16 columns start 256 bytes further on.
//
// Accumulators live in tensor memory: for M = 128, row m is lane m; for
// M = 64, row m is lane (m % 16) + 32 * (m / 16), i.e. the first 16 lanes of
// each warp's quarter. tcgen05.ld.32x32b gives thread t of warp w lane
// 32 w + t.
#pragma once
#include <cstdint>

namespace icm {
namespace tc05 {

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__host__ __device__ constexpr int kmajor_offset(int row, int k, int K)
{
    return ((row >> 3) * (K >> 3) + (k >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

// shared-memory matrix descriptor: K-major, no swizzle
__device__ __forceinline__ uint64_t desc_kmajor(const void *tile, int K)
{
    const uint32_t addr = smem_u32(tile);
    const uint32_t lbo = 128, sbo = (uint32_t)(K >> 3) * 128;
    uint64_t d = (uint64_t)((addr >> 4) & 0x3fff);
    d |= (uint64_t)((lbo >> 4) & 0x3fff) << 16;
    d |= (uint64_t)((sbo >> 4) & 0x3fff) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version of sm_100
    return d;
}

// instruction descriptor: BF16 A and B, FP32 accumulator, both K-major
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// D[tmem] (+)= A * B^T for one K = 16 slice; issued by one thread
__device__ __forceinline__ void mma(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t idesc, bool accumulate)
{
    const uint32_t acc = accumulate ? 1u : 0u, mask = 0u;
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}\n"
        ::"r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"(acc), "r"(mask));
}

// the mbarrier arrives when every MMA issued so far by this thread is done
__device__ __forceinline__ void commit(uint64_t *mbar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar)));
}

__device__ __forceinline__ void mbar_init(uint64_t *mbar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count));
    asm volatile("fence.mbarrier_init.release.cluster;");
}

// Waits for the phase with the given parity; gives up after max_iter polls
// and returns false (the caller records the failure).
__device__ __forceinline__ bool mbar_wait(uint64_t *mbar, uint32_t parity, int max_iter)
{
    uint32_t done = 0;
    for (int it = 0; it < max_iter && !done; it++)
        asm volatile("{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                     "selp.b32 %0, 1, 0, P1;\n\t}\n"
                     : "=r"(done)
                     : "r"(smem_u32(mbar)), "r"(parity));
    return done != 0;
}

// make generic-proxy shared-memory writes visible to the tensor cores
__device__ __forceinline__ void fence_smem_for_mma() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// one warp allocates / frees; ncols a power of two >= 32
__device__ __forceinline__ void alloc(uint32_t *dst_smem, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(dst_smem)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void dealloc(uint32_t tmem, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(ncols));
}

// 16 consecutive FP32 columns of this thread's lane (warp-collective)
__device__ __forceinline__ void ld16(uint32_t taddr, float v[16])
{
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int j = 0; j < 16; j++) v[j] = __uint_as_float(r[j]);
}

// address of column col in the lane quarter of warp w
__device__ __forceinline__ uint32_t taddr(uint32_t base, int warp, int col)
{
    return base + ((uint32_t)(warp * 32) << 16) + (uint32_t)col;
}

}  // namespace tc05
}  // namespace icm
