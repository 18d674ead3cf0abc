// Thin inline-PTX layer over the sm_100a tensor-core path: TMEM allocation,
// UMMA shared-memory / instruction descriptors, tcgen05.mma (kind::f16, BF16
// operands, FP32 accumulate), commit to an mbarrier, TMEM loads and the fences
// that order them. Operand tiles use the no-swizzle canonical layout built
// from 8-row x 16-byte core matrices.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace b200 {
namespace tc {

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory matrix descriptor, no swizzle. `lbo` is the byte stride
// between core matrices along K (K-major) or along the strided dimension
// (MN-major), `sbo` the byte stride between 8-row groups (K-major) or between
// 8-element groups of the contiguous dimension (MN-major).
__device__ __forceinline__ uint64_t desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    uint64_t d = uint64_t((saddr >> 4) & 0x3fffu);
    d |= uint64_t((lbo >> 4) & 0x3fffu) << 16;
    d |= uint64_t((sbo >> 4) & 0x3fffu) << 32;
    d |= uint64_t(1) << 46; // descriptor version of sm_100
    return d;                // base offset 0, layout type 0 (no swizzle)
}

// Instruction descriptor of kind::f16 with BF16 A/B and an FP32 accumulator.
// a_mn / b_mn select MN-major operands (transposed reads of the same tiles).
__host__ __device__ constexpr uint32_t idesc_bf16(uint32_t m, uint32_t n, bool a_mn, bool b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(a_mn) << 15) | (uint32_t(b_mn) << 16) |
           ((n >> 3) << 17) | ((m >> 4) << 24);
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc, uint32_t accum) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
        "l"(a), "l"(b), "r"(idesc), "r"(accum), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void commit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_addr(mbar))
                 : "memory");
}

__device__ __forceinline__ void fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// Makes generic-proxy shared-memory writes visible to the tensor core.
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(mbar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Bounded wait for the phase with parity `parity`; false when it gave up.
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, uint32_t limit) {
    const uint32_t addr = smem_addr(mbar);
    for (uint32_t i = 0; i < limit; ++i) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(addr), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Whole-warp TMEM allocation; the column base is written to *dst (shared).
__device__ __forceinline__ void tmem_alloc(uint32_t* dst, uint32_t columns) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(dst)),
                 "r"(columns)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t base, uint32_t columns) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(base), "r"(columns) : "memory");
}

// Eight consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld8(uint32_t addr, float* out) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    for (int i = 0; i < 8; ++i) out[i] = __uint_as_float(r[i]);
}

// Byte offset of element (row, k) in a K-major no-swizzle tile whose K extent
// is `kext` elements of 2 bytes: core matrices of 8 rows x 16 bytes, K-chunks
// 128 bytes apart, 8-row groups kext * 16 bytes apart.
__host__ __device__ constexpr uint32_t kmajor_offset(uint32_t row, uint32_t k, uint32_t kext) {
    return (row >> 3) * (kext * 16) + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

} // namespace tc
} // namespace b200
