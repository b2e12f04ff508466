// tcgen05 (5th-generation tensor core) primitives for sm_100a: TMEM
// allocation, shared-memory matrix descriptors for K-major BF16 tiles without
// swizzle, the kind::f16 MMA with an FP32 accumulator in TMEM, commit to an
// mbarrier, bounded waits and TMEM loads.
//
// Shared-memory tile layout ("core matrices", no swizzle, K-major): a tile
// of R rows x K bf16 columns (R multiple of 8, K multiple of 8) is stored as
// 8-row x 16-byte core matrices; element (r, k) lives at
//   (r / 8) * SBO + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2   bytes,
// with the K chunks of one row group adjacent (leading byte offset 128) and
// row groups SBO = K / 8 * 128 bytes apart.
#pragma once
#include <cstdint>
#include <cuda_bf16.h>

namespace smb {
namespace umma {

__device__ __forceinline__ uint32_t saddr(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

__host__ __device__ constexpr uint32_t tile_offset(uint32_t r, uint32_t k, uint32_t K) {
    return (r / 8) * (K / 8) * 128 + (k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2;
}

// Descriptor of the K-major no-swizzle tile at smem byte address `addr`,
// K columns wide (one MMA reads 16 of them starting at `addr`).
__device__ __forceinline__ uint64_t desc_kmajor(uint32_t addr, uint32_t K) {
    const uint64_t lbo = 128, sbo = uint64_t(K / 8) * 128;
    return uint64_t((addr >> 4) & 0x3FFF) | ((lbo >> 4) << 16) | ((sbo >> 4) << 32) | (uint64_t(1) << 46);
}

// Instruction descriptor: D f32, A and B bf16, both K-major, shape M x N.
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t M, uint32_t N) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((N >> 3) << 17) | ((M >> 4) << 24);
}

__device__ __forceinline__ void tmem_alloc(uint32_t* dst_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(saddr(dst_smem)), "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Generic-proxy shared-memory writes made visible to the tensor core.
__device__ __forceinline__ void fence_smem_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// D[tmem] (+)= A[smem] * B[smem]^T, issued by one thread.
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
    uint32_t mask0 = 0, mask1 = 0, mask2 = 0, mask3 = 0;
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(mask0), "r"(mask1), "r"(mask2), "r"(mask3));
}

// Arrives once on the mbarrier when every MMA issued so far has completed.
__device__ __forceinline__ void commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(saddr(bar))
                 : "memory");
}

__device__ __forceinline__ void bar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(saddr(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for a phase of the mbarrier; false if it gave up.
__device__ __forceinline__ bool bar_wait(uint64_t* bar, uint32_t parity, uint32_t limit = 1u << 24) {
    for (uint32_t i = 0; i < limit; i++) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(saddr(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// This warp's 32 TMEM lanes (rows 32 * (warp % 4) + lane), 8 consecutive
// 32-bit columns starting at `col`.
__device__ __forceinline__ void ld8(uint32_t tmem_base, uint32_t warp, uint32_t col, float v[8]) {
    uint32_t a = tmem_base + ((32u * (warp & 3u)) << 16) + col;
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(a));
    for (int i = 0; i < 8; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void ld_wait() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

}  // namespace umma
}  // namespace smb
