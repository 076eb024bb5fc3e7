// sph_tc.cuh -- the pieces of Blackwell's 5th-generation tensor-core path
// (tcgen05) that the smoothing-length MLP uses: shared-memory matrix
// descriptors, the instruction descriptor of a BF16 x BF16 -> FP32 MMA, the
// MMA issue, its completion through an mbarrier (bounded wait), tensor-memory
// (TMEM) allocation and loads.  Inline PTX for sm_100a.
//
// Operands live in shared memory in the canonical K-major layout without
// swizzle: 8 x 16-byte "core matrices" (8 rows x 8 BF16 values along K),
//   byte offset (row, k) = (row / 8) * SBO + (k / 8) * LBO + (row % 8) * 16 + (k % 8) * 2,
// with LBO = 128 (the K-adjacent core matrix) and SBO = (K / 8) * 128.
// One MMA consumes a K = 16 slice, starting (k0 / 8) * 128 bytes in.
#pragma once

#include <cuda_bf16.h>
#include <cstdint>

namespace sph {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Byte offset of element (row, k) of a K-major operand with K columns.
__device__ __forceinline__ uint32_t kmajor_off(int row, int k, int K) {
    return (uint32_t)((row >> 3) * (K >> 3) * 128 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

// Shared-memory matrix descriptor, K-major, no swizzle (layout type 0),
// descriptor version 1.
__device__ __forceinline__ uint64_t kmajor_desc(uint32_t start, int K) {
    const uint64_t lbo = 128u >> 4, sbo = (uint64_t)((K >> 3) * 128) >> 4;
    return (uint64_t)((start >> 4) & 0x3fffu) | (lbo << 16) | (sbo << 32) | (1ull << 46);
}

// Instruction descriptor: D FP32, A and B BF16, both K-major, M = 128, N.
__host__ __device__ constexpr uint32_t idesc_bf16_m128(int N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

// D[tmem] (+)= A * B^T for one K = 16 slice; issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         bool accumulate) {
    const uint32_t acc = accumulate ? 1u : 0u, z = 0u;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(acc), "r"(z), "r"(z), "r"(z), "r"(z));
}

// Arrive on the mbarrier when every MMA issued so far by this thread is done.
__device__ __forceinline__ void mma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Wait for the phase with the given parity to complete, polling at most
// `limit` times; returns false when the wait gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int limit) {
    const uint32_t a = smem_u32(bar);
    for (int i = 0; i < limit; ++i) {
        uint32_t done = 0;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Make generic-proxy writes to shared memory visible to the tensor core.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

// TMEM allocation (one warp, warp-wide); the base address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t base, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(ncols) : "memory");
}

// 16 consecutive FP32 columns of this thread's TMEM lane (warp w reads lanes
// 32w..32w+31; addr carries lane << 16 | column).
__device__ __forceinline__ void tmem_ld16(uint32_t addr, float *v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace tc
}  // namespace sph
