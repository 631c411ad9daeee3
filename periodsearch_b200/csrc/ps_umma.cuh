// tcgen05 (5th-generation tensor core) building blocks for sm_100a: TMEM
// allocation, shared-memory matrix descriptors, BF16 MMA issue, commit to an
// mbarrier, TMEM loads, and bounded mbarrier waits.  Inline PTX, one
// CTA (cta_group::1), no clusters and no multicast.
//
// Operand layout: K-major with the 128-byte swizzle.  A tile of R rows and
// 64 BF16 along K occupies R*128 bytes; row r, element k lives at byte
//   r*128 + ((2k) ^ ((r & 7) << 4))
// (16-byte chunks XOR-ed with the row index mod 8), tile bases 1024-byte
// aligned.  Descriptor: start address >> 4, LBO = 1 (unused for swizzled
// K-major), SBO = 1024 B (distance between 8-row groups), version 1,
// layout SWIZZLE_128B (= 2); one UMMA_K = 16 BF16 = 32 bytes, so k-step kk
// of a 64-wide tile starts 32*kk bytes in.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace psb {
namespace umma {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t desc_kmajor_sw128(uint32_t saddr) {
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)1u << 16;            // LBO (unused)
    d |= (uint64_t)(1024u >> 4) << 32;  // SBO = 1024 bytes
    d |= (uint64_t)1u << 46;            // descriptor version for sm_100
    d |= (uint64_t)2u << 61;            // SWIZZLE_128B
    return d;
}

// Instruction descriptor, kind::f16 with BF16 A/B, FP32 D, both K-major.
__host__ __device__ constexpr uint32_t idesc_bf16_f32(int M, int N) {
    return (1u << 4)                  // D format F32
           | (1u << 7)                // A format BF16
           | (1u << 10)               // B format BF16
           | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Instruction descriptor, kind::tf32 with TF32 A/B (FP32 storage, the top 19
// bits used), FP32 D, both K-major.  A 128-byte K row holds 32 elements, one
// MMA step (UMMA_K = 8) 32 bytes: the same descriptors and k-step offsets as
// the BF16 tiles.
__host__ __device__ constexpr uint32_t idesc_tf32_f32(int M, int N) {
    return (1u << 4)                  // D format F32
           | (2u << 7)                // A format TF32
           | (2u << 10)               // B format TF32
           | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// byte offset of element (r, k) in a K-major SW128 FP32 tile (32 wide)
__device__ __forceinline__ uint32_t sw128_off32(int r, int k) {
    return (uint32_t)(r * 128) + ((uint32_t)(4 * k) ^ ((uint32_t)(r & 7) << 4));
}

// byte offset of element (r, k) in a K-major SW128 BF16 tile (64 wide)
__device__ __forceinline__ uint32_t sw128_off(int r, int k) {
    return (uint32_t)(r * 128) + ((uint32_t)(2 * k) ^ ((uint32_t)(r & 7) << 4));
}

// TMEM allocation by one full warp; the base address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate));
}

// Arrive on the mbarrier once every tcgen05 operation issued so far by this
// thread has completed.
__device__ __forceinline__ void commit(uint64_t* mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(mbar))
                 : "memory");
}

__device__ __forceinline__ void mbar_init(uint64_t* mbar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(count));
}

// Wait for the phase with the given parity to complete; gives up after
// max_polls polls and returns false (the caller records the failure).
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity, uint32_t max_polls) {
    const uint32_t a = smem_u32(mbar);
    for (uint32_t i = 0; i < max_polls; i++) {
        uint32_t done;
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\nselp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(a), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// 32 lanes x 32 bits, 16 consecutive columns per thread.  The load and its
// wait are one asm statement, so no use of the destination registers can be
// scheduled between them.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

// FP32 -> (hi, lo) TF32 pair (FP32 bit patterns with the low 13 bits zero,
// round to nearest) with x ~= hi + lo to ~2^-22 relative.
__device__ __forceinline__ void split_tf32(float x, uint32_t& hi, uint32_t& lo) {
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(x));
    const float r = x - __uint_as_float(hi);
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"(r));
}

// FP32 -> (hi, lo) BF16 pair with x ~= hi + lo to ~2^-16 relative.
__device__ __forceinline__ void split_bf16(float x, __nv_bfloat16& hi, __nv_bfloat16& lo) {
    hi = __float2bfloat16_rn(x);
    lo = __float2bfloat16_rn(x - __bfloat162float(hi));
}

}  // namespace umma
}  // namespace psb
