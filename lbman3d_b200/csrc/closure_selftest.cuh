// closure_selftest.cuh -- a single-CTA tcgen05 GEMM, D[128 x N] = A[128 x K]
// * B[N x K]^T with BF16 operands staged in either major order, used to
// check the descriptor / layout conventions of tc.cuh on the device before
// the convolution kernels rely on them.
#pragma once

#include "tc.cuh"

namespace lbman {

constexpr int kSelfM = 128, kSelfN = 32, kSelfK = 64;
// A at offset 0, B at 48 KB: every stride interpretation of either
// descriptor stays inside the 64 KB of dynamic shared memory.
constexpr uint32_t kSelfBOff = 48 * 1024;
constexpr uint32_t kSelfSmem = 64 * 1024;

__global__ void __launch_bounds__(128) tc_selftest_kernel(const float* __restrict__ A, const float* __restrict__ B,
                                                          float* __restrict__ D, int a_mn, int b_mn,
                                                          int* __restrict__ err) {
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ uint64_t bar;
    __shared__ uint32_t tslot;
    const int t = threadIdx.x;
    // operand strides (bytes): K-major rows-then-k, MN-major k-then-rows
    const uint32_t a_lbo = a_mn ? (kSelfM / 8) * 128 : 128, a_sbo = a_mn ? 128 : (kSelfK / 8) * 128;
    const uint32_t b_lbo = b_mn ? (kSelfN / 8) * 128 : 128, b_sbo = b_mn ? 128 : (kSelfK / 8) * 128;
    for (int i = t; i < kSelfM * kSelfK; i += blockDim.x) {
        const int r = i / kSelfK, k = i % kSelfK;
        const uint32_t o = a_mn ? tc::mnmajor_off(r, k, a_lbo, a_sbo) : tc::kmajor_off(r, k, a_lbo, a_sbo);
        *reinterpret_cast<__nv_bfloat16*>(sm + o) = __float2bfloat16(A[i]);
    }
    for (int i = t; i < kSelfN * kSelfK; i += blockDim.x) {
        const int r = i / kSelfK, k = i % kSelfK;
        const uint32_t o = b_mn ? tc::mnmajor_off(r, k, b_lbo, b_sbo) : tc::kmajor_off(r, k, b_lbo, b_sbo);
        *reinterpret_cast<__nv_bfloat16*>(sm + kSelfBOff + o) = __float2bfloat16(B[i]);
    }
    if (t == 0) {
        tc::mbar_init(&bar, 1);
        tc::mbar_fence_init();
    }
    if (t < 32) tc::tmem_alloc(&tslot, 32);
    tc::fence_smem_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tslot;
    if (t == 0) {
        const uint32_t id = tc::idesc_bf16(kSelfM, kSelfN, a_mn, b_mn);
        const uint32_t a0 = tc::smem_addr(sm), b0 = tc::smem_addr(sm + kSelfBOff);
#pragma unroll
        for (int j = 0; j < kSelfK / 16; ++j) {
            const uint64_t da = tc::smem_desc(a0 + j * 2 * a_lbo, a_lbo, a_sbo);
            const uint64_t db = tc::smem_desc(b0 + j * 2 * b_lbo, b_lbo, b_sbo);
            tc::mma_bf16(tmem, da, db, id, j > 0 ? 1u : 0u);
        }
        tc::mma_commit(&bar);
    }
    const bool ok = tc::mbar_wait(&bar, 0, err);
    tc::fence_after_sync();
    if (ok) {
        const int w = t >> 5, lane = t & 31;
        const int row = 32 * w + lane;
#pragma unroll
        for (int c0 = 0; c0 < kSelfN; c0 += 16) {
            float v[16];
            tc::tmem_ld16(tmem + ((uint32_t)(32 * w) << 16) + (uint32_t)c0, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) D[row * kSelfN + c0 + i] = v[i];
        }
    }
    tc::fence_before_sync();
    __syncthreads();
    if (t < 32) tc::tmem_dealloc(tmem, 32);
}

}  // namespace lbman
