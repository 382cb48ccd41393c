// tc.cuh -- fifth-generation tensor-core (tcgen05) building blocks for the
// closure network's BF16 convolutions on sm_100a: TMEM allocation, shared
// memory matrix descriptors (no swizzle), the kind::f16 MMA issued by one
// thread, completion through an mbarrier, and TMEM -> register loads.
//
// Shared-memory operand layout (SWIZZLE_NONE, 16-bit elements).  An operand
// of R rows (M or N) by 16 K-elements is a grid of 8x8 "core matrices", each
// 128 contiguous bytes:
//   K-major : core (r/8, k/8) holds rows r%8 at 16-byte pitch, 8 consecutive
//             k of one row in each 16 bytes;
//   MN-major: core (r/8, k/8) holds k%8 at 16-byte pitch, 8 consecutive rows
//             of one k in each 16 bytes.
// byte(r, k) = (r/8)*SBO + (k/8)*LBO + (K-major ? (r%8)*16 + (k%8)*2
//                                               : (k%8)*16 + (r%8)*2).
// The descriptor carries start>>4, LBO>>4 (bits 16-29), SBO>>4 (32-45) and
// the sm_100 version bit 46; swizzle mode 0.
//
// Every wait is bounded: a wait that gives up sets *err and returns, so a
// kernel never spins forever.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

namespace lbman {
namespace tc {

constexpr uint32_t kWaitLimit = 1u << 26;  // polls before a wait gives up

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

__host__ __device__ constexpr uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}

// kind::f16 instruction descriptor: BF16 A and B, FP32 accumulator, M x N,
// operand majors (0 = K-major, 1 = MN-major).
__host__ __device__ constexpr uint32_t idesc_bf16(int M, int N, int a_mn, int b_mn) {
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)b_mn << 16) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// byte offset of element (r, k) inside an operand laid out as above
__host__ __device__ constexpr uint32_t kmajor_off(int r, int k, uint32_t lbo, uint32_t sbo) {
    return (uint32_t)(r / 8) * sbo + (uint32_t)(k / 8) * lbo + (uint32_t)(r % 8) * 16u + (uint32_t)(k % 8) * 2u;
}
__host__ __device__ constexpr uint32_t mnmajor_off(int r, int k, uint32_t lbo, uint32_t sbo) {
    return (uint32_t)(r / 8) * sbo + (uint32_t)(k / 8) * lbo + (uint32_t)(k % 8) * 16u + (uint32_t)(r % 8) * 2u;
}

// --- TMEM allocation (one warp, all lanes) --------------------------------
__device__ __forceinline__ void tmem_alloc(uint32_t* slot_smem, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot_smem)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols));
}

// --- ordering ----------------------------------------------------------------
__device__ __forceinline__ void fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
// generic-proxy shared-memory writes -> visible to the tensor core (async proxy)
__device__ __forceinline__ void fence_smem_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// --- mbarrier -------------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_fence_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return done != 0;
}
// Bounded wait for the phase with this parity; false (and *err set) if it
// did not complete within `limit` polls (0: give up without polling).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, uint32_t limit = kWaitLimit) {
    for (uint32_t i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    if (err) atomicExch(err, 1);
    return false;
}

// --- MMA (issued by one thread) -------------------------------------------
__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc,
                                         uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred P;\n\t"
        "setp.ne.b32 P, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, P;\n\t}"
        :
        : "r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(accumulate)
        : "memory");
}
// Arrive on bar once every MMA this thread issued so far has completed.
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_addr(bar))
                 : "memory");
}

// --- TMEM -> registers: warp w reads lanes [32w, 32w+32), thread = lane -----
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float v[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_ld8(uint32_t taddr, float v[8]) {
    uint32_t r[8];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace tc
}  // namespace lbman
