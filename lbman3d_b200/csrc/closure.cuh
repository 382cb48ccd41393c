// closure.cuh -- kernels of the learned closure: a 4-layer 3x3x3 periodic
// convolutional network (9 -> 32 -> 32 -> 32 -> 8 channels, GELU after the
// first three layers) on a coarse grid, with BF16 operands on the tcgen05
// tensor cores and FP32 accumulation in TMEM.  No counterpart in the
// reference.
//
// Activations are channel-last BF16, act[cell][C] with C = 16 (the 9 input
// features, zero padded) or 32; the last layer's 8 outputs are padded to 16.
// A convolution is an implicit GEMM: for a tile of 128 cells (M) and each of
// the 27 taps, the 128 x CIN neighbour rows are gathered into shared memory
// (K-major) and multiplied by that tap's CIN x COUT weights (N = COUT), all
// 27 taps accumulating into one TMEM accumulator.  Two A stages let the
// gather of tap t+1 overlap the MMAs of tap t.  The backward data pass is
// the same kernel run with the transposed, tap-reversed weight image; the
// weight gradient is a GEMM over cells (K) with M = (tap, ci) rows and
// MN-major operands taken straight from the channel-last activations.
//
// Tap index: tap = (dz+1)*9 + (dy+1)*3 + (dx+1); output cell c reads input
// cell c + (dx, dy, dz) with periodic wrap on every axis.
//
// Waits: every wait for MMA completion that the pipeline needs to go on
// polls at most wait_limit times (a kernel argument; tc::kWaitLimit unless
// the caller lowered it).  A wait that gives up sets *err, the whole CTA
// leaves its tile loop together (__syncthreads_or), and the drain waits --
// always with the full tc::kWaitLimit, because the tensor core must finish
// every MMA it was given before the CTA frees its TMEM -- end the kernel.
#pragma once

#include <cuda_bf16.h>
#include <stdint.h>

#include "tc.cuh"

namespace lbman {
namespace cl {

constexpr int kTileM = 128;
constexpr int kThreads = 128;
constexpr int kStages = 4;  // A-operand stages of the convolution pipeline

struct Grid3 {
    int nx, ny, nz;
    int64_t V;
};

__device__ __forceinline__ int wrapi(int a, int n) { return a < 0 ? a + n : (a >= n ? a - n : a); }

__device__ __forceinline__ int64_t neighbour(const Grid3& g, int x, int y, int z, int tap) {
    const int dx = tap % 3 - 1, dy = (tap / 3) % 3 - 1, dz = tap / 9 - 1;
    return ((int64_t)wrapi(z + dz, g.nz) * g.ny + wrapi(y + dy, g.ny)) * g.nx + wrapi(x + dx, g.nx);
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
    const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
    return cdf + x * pdf;
}

// Byte size of the B image of one convolution: 27 taps x CIN/16 k-steps of
// COUT x 16 K-major BF16 (core matrices: n-group stride 256, k-group 128).
__host__ __device__ constexpr int bimg_bytes(int cin, int cout) { return 27 * (cin / 16) * cout * 32; }

enum ConvMode : int {
    kFwdHidden = 0,  // + bias, store pre (BF16) and GELU(pre) (BF16)
    kFwdLast = 1,    // + bias, store FP32
    kBwdData = 2     // times GELU'(pre of the layer below), store BF16
};

// Halo staging applies when a 128-cell tile is R = 128/nx whole x rows of
// one z plane: then the tile's input neighbourhood (3 planes x R+2 rows x nx
// cells) is copied into shared memory once per tile and the 27 tap operands
// are built from it, instead of 27 gathers from L2.
__host__ __device__ inline bool halo_ok(int nx, int ny) {
    return nx <= kTileM && kTileM % nx == 0 && ((int64_t)nx * ny) % kTileM == 0;
}
__host__ __device__ inline int halo_bytes(int nx, int cin) { return 3 * (kTileM / nx + 2) * nx * cin * 2; }

// One persistent CTA walks 128-cell tiles.  Smem: B image, kStages A stages
// of CIN/16 x 4 KB, then (halo != 0) the staged neighbourhood.  The operand
// of tap k goes to stage k % kStages once the MMAs that last read that stage
// have completed, so operand copies run up to kStages - 1 taps ahead of the
// tensor core.  Halo units of
// 16 bytes are stored at cell * (CIN/8) + (q ^ (cell & (CIN/8 - 1))), an XOR
// swizzle that spreads a warp's reads of one q over the banks.
template <int CIN, int COUT, int MODE>
__global__ void __launch_bounds__(kThreads) conv_kernel(Grid3 g, const __nv_bfloat16* __restrict__ in,
                                                        const uint4* __restrict__ bimg, const float* __restrict__ bias,
                                                        const __nv_bfloat16* __restrict__ pre_below,
                                                        __nv_bfloat16* __restrict__ out_pre,
                                                        __nv_bfloat16* __restrict__ out_bf, float* __restrict__ out_f,
                                                        int halo, int* __restrict__ err,
        uint32_t wait_limit) {
    constexpr int KS = CIN / 16;                 // k-steps per tap
    constexpr int BBYTES = bimg_bytes(CIN, COUT);
    constexpr int ABYTES = KS * 4096;            // one A stage
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ uint64_t bar[kStages];
    __shared__ uint32_t tslot;
    constexpr int QU = CIN / 8;                  // 16-byte units per cell
    unsigned char* Bs = sm;
    unsigned char* As = sm + BBYTES;
    uint4* Hs = reinterpret_cast<uint4*>(sm + BBYTES + kStages * ABYTES);
    const int t = threadIdx.x;
    const int R = kTileM / g.nx;                 // rows per tile (halo path)

    for (int i = t; i < BBYTES / 16; i += kThreads) reinterpret_cast<uint4*>(Bs)[i] = bimg[i];
    if (t == 0) {
        for (int k = 0; k < kStages; ++k) tc::mbar_init(&bar[k], 1);
        tc::mbar_fence_init();
    }
    if (t < 32) tc::tmem_alloc(&tslot, 32);
    tc::fence_smem_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tslot;
    const uint32_t idesc = tc::idesc_bf16(kTileM, COUT, 0, 0);
    const uint32_t a0 = tc::smem_addr(As), b0 = tc::smem_addr(Bs);
    uint32_t uses[kStages] = {};  // commits issued per A stage (same in every thread)
    int kt = 0;                     // taps issued so far by this CTA
    int last_s = 0;
    bool ok = true;

    const int64_t ntiles = (g.V + kTileM - 1) / kTileM;
    for (int64_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int64_t c = tile * kTileM + t;
        const bool live = c < g.V;
        const int64_t cc = live ? c : 0;
        const int x = (int)(cc % g.nx), y = (int)((cc / g.nx) % g.ny), z = (int)(cc / ((int64_t)g.nx * g.ny));
        if (halo) {
            // planes z0-1..z0+1, rows y0-1..y0+R of the tile's plane
            const int64_t c0 = tile * kTileM;
            const int z0 = (int)(c0 / ((int64_t)g.nx * g.ny)), y0 = (int)((c0 / g.nx) % g.ny);
            const int nunits = 3 * (R + 2) * g.nx * QU;
            for (int i = t; i < nunits; i += kThreads) {
                const int q = i % QU, cell = i / QU;
                const int hx = cell % g.nx, hr = (cell / g.nx) % (R + 2), hz = cell / (g.nx * (R + 2));
                const int64_t src = ((int64_t)wrapi(z0 - 1 + hz, g.nz) * g.ny + wrapi(y0 - 1 + hr, g.ny)) * g.nx + hx;
                const uint4* gp = reinterpret_cast<const uint4*>(in + src * CIN) + q;
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(
                                 tc::smem_addr(Hs + cell * QU + (q ^ (cell & (QU - 1))))),
                             "l"(gp));
            }
            asm volatile("cp.async.wait_all;\n" ::: "memory");
            __syncthreads();
        }
        for (int tap = 0; tap < 27; ++tap, ++kt) {
            const int s = kt % kStages;
            // stage s is free once the MMAs that read it last have completed
            bool lost = uses[s] > 0 && !tc::mbar_wait(&bar[s], (uses[s] - 1) & 1, err, wait_limit);
            if (__syncthreads_or(lost)) {
                ok = false;
                break;
            }
            // this row's CIN channels of the neighbour into stage s
            unsigned char* dst = As + s * ABYTES + (t / 8) * 256 + (t % 8) * 16;
            if (halo) {
                const int dx = tap % 3 - 1, dy = (tap / 3) % 3 - 1, dz = tap / 9 - 1;
                const int hx = wrapi(t % g.nx + dx, g.nx), hr = t / g.nx + 1 + dy;
                const int cell = ((1 + dz) * (R + 2) + hr) * g.nx + hx;
#pragma unroll
                for (int q = 0; q < QU; ++q)
                    *reinterpret_cast<uint4*>(dst + (q / 2) * 4096 + (q % 2) * 128) =
                        Hs[cell * QU + (q ^ (cell & (QU - 1)))];
            } else {
                const uint4* src = reinterpret_cast<const uint4*>(in + neighbour(g, x, y, z, tap) * CIN);
#pragma unroll
                for (int q = 0; q < QU; ++q)
                    *reinterpret_cast<uint4*>(dst + (q / 2) * 4096 + (q % 2) * 128) = src[q];
            }
            tc::fence_smem_async();
            tc::fence_before_sync();
            __syncthreads();
            tc::fence_after_sync();
            if (t == 0) {
#pragma unroll
                for (int kb = 0; kb < KS; ++kb) {
                    const uint64_t da = tc::smem_desc(a0 + s * ABYTES + kb * 4096, 128, 256);
                    const uint64_t db = tc::smem_desc(b0 + (tap * KS + kb) * COUT * 32, 128, 256);
                    tc::mma_bf16(tmem, da, db, idesc, (tap > 0 || kb > 0) ? 1u : 0u);
                }
                tc::mma_commit(&bar[s]);
            }
            ++uses[s];
            last_s = s;
        }
        if (!ok) break;
        // the tile's last commit covers every MMA issued before it
        const bool lost = !tc::mbar_wait(&bar[last_s], (uses[last_s] - 1) & 1, err, wait_limit);
        if (__syncthreads_or(lost)) {
            ok = false;
            break;
        }
        tc::fence_after_sync();
        const int w = t >> 5;
        float acc[COUT];
#pragma unroll
        for (int c0 = 0; c0 < COUT; c0 += 16) tc::tmem_ld16(tmem + ((uint32_t)(32 * w) << 16) + (uint32_t)c0, acc + c0);
        if (live) {
            if constexpr (MODE == kFwdHidden) {
                __align__(16) __nv_bfloat16 pb[COUT], ab[COUT];
#pragma unroll
                for (int j = 0; j < COUT; ++j) {
                    const float p = acc[j] + bias[j];
                    pb[j] = __float2bfloat16(p);
                    ab[j] = __float2bfloat16(gelu(p));
                }
#pragma unroll
                for (int q = 0; q < COUT / 8; ++q) {
                    reinterpret_cast<uint4*>(out_pre + c * COUT)[q] = reinterpret_cast<const uint4*>(pb)[q];
                    reinterpret_cast<uint4*>(out_bf + c * COUT)[q] = reinterpret_cast<const uint4*>(ab)[q];
                }
            } else if constexpr (MODE == kFwdLast) {
#pragma unroll
                for (int j = 0; j < COUT; j += 4)
                    reinterpret_cast<float4*>(out_f + c * COUT)[j / 4] =
                        make_float4(acc[j] + bias[j], acc[j + 1] + bias[j + 1], acc[j + 2] + bias[j + 2],
                                    acc[j + 3] + bias[j + 3]);
            } else {
                __align__(16) __nv_bfloat16 pre[COUT], gb[COUT];
#pragma unroll
                for (int q = 0; q < COUT / 8; ++q)
                    reinterpret_cast<uint4*>(pre)[q] = reinterpret_cast<const uint4*>(pre_below + c * COUT)[q];
#pragma unroll
                for (int j = 0; j < COUT; ++j) gb[j] = __float2bfloat16(acc[j] * gelu_grad(__bfloat162float(pre[j])));
#pragma unroll
                for (int q = 0; q < COUT / 8; ++q)
                    reinterpret_cast<uint4*>(out_bf + c * COUT)[q] = reinterpret_cast<const uint4*>(gb)[q];
            }
        }
        tc::fence_before_sync();
        __syncthreads();  // TMEM reads done before the next tile's first MMA
        tc::fence_after_sync();
    }
    // drain: never leave with MMAs in flight on our TMEM
    if (t == 0) {
        for (int s = 0; s < kStages; ++s)
            if (uses[s] > 0) tc::mbar_wait(&bar[s], (uses[s] - 1) & 1, err);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (t < 32) tc::tmem_dealloc(tmem, 32);
}

// ---- descriptor-halo convolution, z-marching ---------------------------------
// Tile = 8 x-cells by 16 y-rows of one z plane (128 cells, M row m = 8*dy_row
// + dx_cell).  A CTA takes a column of tiles (the same 8 x 16 block of every
// plane of a z range) and marches it in z.  The column's neighbourhood is
// staged plane by plane (10 x 18 cells per plane) in a ring of 5 plane slots,
// as 16-byte units, one block per 8-channel group:
//   unit(slot, kg, hy, hx) at slot*SLOT + (kg*18 + hy)*10 + hx,
// which makes the A operand of every tap a K-major view of the ring: rows of
// a core matrix are 8 consecutive x cells (16 bytes apart), the next y row is
// SBO = 160 bytes on, the next 8 channels LBO = 2880 bytes on, and the tap
// (dx, dy, dz) only picks the slot of plane z + dz and moves the start
// address.  So each tile costs one new plane (the other two are the previous
// tiles') and 27 x CIN/16 back-to-back MMAs with no operand copies; the copy
// of a plane is issued two tiles before the tile that first reads it.  The
// TMEM accumulator is double buffered.  Warps 0-7 copy planes and run the
// epilogues (warps w and w + 4 read the same TMEM lanes, 32 (w % 4) ..,
// and split the accumulator's columns); warp 8 issues the MMAs.  So while
// the tensor core runs tile z, warps 0-7 start copying plane z + 3, finish
// tile z - 1 and wait for plane z + 2, and warp 8 has queued tile z: one
// block barrier per tile.
constexpr int kHX = 10, kHY = 18;
constexpr int kZWorkers = 256;             // copy / epilogue threads
constexpr int kZThreads = kZWorkers + 32;  // + the MMA warp
constexpr int kZIssuer = kZWorkers;        // the thread that issues the MMAs
constexpr int kSlots = 5;
__host__ __device__ constexpr int ring_slot(int plane) { return (plane + kSlots) % kSlots; }  // plane >= -1
__host__ __device__ constexpr int dhalo_slot_bytes(int cin) { return (cin / 8) * kHX * kHY * 16; }
__host__ __device__ constexpr int dhalo_bytes(int cin) { return kSlots * dhalo_slot_bytes(cin); }

__host__ __device__ inline bool dhalo_ok(int nx, int ny) { return nx % 8 == 0 && ny % 16 == 0; }

// Copies plane zz (-1 <= zz <= nz, periodic) of the column at (x0, y0) into
// its ring slot S (worker threads).
template <int CIN>
__device__ __forceinline__ void dhalo_load_plane(const Grid3& g, const __nv_bfloat16* __restrict__ in, int x0,
                                                 int y0, int zz, unsigned char* S) {
    constexpr int N = (CIN / 8) * kHX * kHY;
    const int64_t zoff = (int64_t)wrapi(zz, g.nz) * g.ny;
    for (int i = threadIdx.x; i < N; i += kZWorkers) {
        const int hx = i % kHX, hy = (i / kHX) % kHY, kg = i / (kHX * kHY);
        const int64_t cell = (zoff + wrapi(y0 - 1 + hy, g.ny)) * g.nx + wrapi(x0 - 1 + hx, g.nx);
        const uint4* src = reinterpret_cast<const uint4*>(in + cell * CIN) + kg;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(tc::smem_addr(S + i * 16)), "l"(src));
    }
}

// Epilogue of one tile: this thread's cell c (TMEM lane = threadIdx % 128)
// and its half of the COUT accumulator columns (bias: that half's biases).
template <int COUT, int MODE>
__device__ __forceinline__ void conv_epilogue(uint32_t tacc, int64_t c, const float (&bias)[COUT / 2],
                                              const __nv_bfloat16* __restrict__ pre_below,
                                              __nv_bfloat16* __restrict__ out_pre, __nv_bfloat16* __restrict__ out_bf,
                                              float* __restrict__ out_f) {
    constexpr int H = COUT / 2;
    static_assert(H == 8 || H == 16, "16 or 32 output channels");
    const int w = threadIdx.x >> 5, half = threadIdx.x >> 7;
    const int j0 = half * H;
    float acc[H];
    const uint32_t ta = tacc + ((uint32_t)(32 * (w & 3)) << 16) + (uint32_t)j0;
    if constexpr (H == 16) tc::tmem_ld16(ta, acc);
    else tc::tmem_ld8(ta, acc);
    if constexpr (MODE == kFwdHidden) {
        __align__(16) __nv_bfloat16 pb[H], ab[H];
#pragma unroll
        for (int j = 0; j < H; ++j) {
            const float p = acc[j] + bias[j];
            pb[j] = __float2bfloat16(p);
            ab[j] = __float2bfloat16(gelu(p));
        }
#pragma unroll
        for (int q = 0; q < H / 8; ++q) {
            reinterpret_cast<uint4*>(out_pre + c * COUT + j0)[q] = reinterpret_cast<const uint4*>(pb)[q];
            reinterpret_cast<uint4*>(out_bf + c * COUT + j0)[q] = reinterpret_cast<const uint4*>(ab)[q];
        }
    } else if constexpr (MODE == kFwdLast) {
#pragma unroll
        for (int j = 0; j < H; j += 4)
            reinterpret_cast<float4*>(out_f + c * COUT + j0)[j / 4] =
                make_float4(acc[j] + bias[j], acc[j + 1] + bias[j + 1], acc[j + 2] + bias[j + 2],
                            acc[j + 3] + bias[j + 3]);
    } else {
        __align__(16) __nv_bfloat16 pre[H], gb[H];
#pragma unroll
        for (int q = 0; q < H / 8; ++q)
            reinterpret_cast<uint4*>(pre)[q] = reinterpret_cast<const uint4*>(pre_below + c * COUT + j0)[q];
#pragma unroll
        for (int j = 0; j < H; ++j) gb[j] = __float2bfloat16(acc[j] * gelu_grad(__bfloat162float(pre[j])));
#pragma unroll
        for (int q = 0; q < H / 8; ++q)
            reinterpret_cast<uint4*>(out_bf + c * COUT + j0)[q] = reinterpret_cast<const uint4*>(gb)[q];
    }
}

// Block b marches column b % cols over planes [zc * (b / cols), + zc).
// Smem: B image, then the plane ring.  TMEM: two 32-column accumulators.
template <int CIN, int COUT, int MODE>
__global__ void __launch_bounds__(kZThreads) conv_dhalo_kernel(Grid3 g, int zc, const __nv_bfloat16* __restrict__ in,
                                                               const uint4* __restrict__ bimg,
                                                               const float* __restrict__ bias,
                                                               const __nv_bfloat16* __restrict__ pre_below,
                                                               __nv_bfloat16* __restrict__ out_pre,
                                                               __nv_bfloat16* __restrict__ out_bf,
                                                               float* __restrict__ out_f, int* __restrict__ err,
                                                               uint32_t wait_limit) {
    constexpr int KS = CIN / 16;
    constexpr int BBYTES = bimg_bytes(CIN, COUT);
    constexpr int SLOT = dhalo_slot_bytes(CIN);
    constexpr uint32_t KG = kHX * kHY;  // 16-byte units between 8-channel groups
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ uint64_t bar[2];
    __shared__ uint32_t tslot;
    unsigned char* Bs = sm;
    unsigned char* Hs = sm + BBYTES;
    const int t = threadIdx.x;
    for (int i = t; i < BBYTES / 16; i += kZThreads) reinterpret_cast<uint4*>(Bs)[i] = bimg[i];
    if (t == 0) {
        tc::mbar_init(&bar[0], 1);
        tc::mbar_init(&bar[1], 1);
        tc::mbar_fence_init();
    }
    if (t < 32) tc::tmem_alloc(&tslot, 64);
    const int bx = g.nx / 8, cols = bx * (g.ny / 16);
    const int col = (int)(blockIdx.x % (unsigned)cols);
    const int x0 = (col % bx) * 8, y0 = (col / bx) * 16;
    const int za = (int)(blockIdx.x / (unsigned)cols) * zc, zb = min(za + zc, g.nz);
    const bool worker = t < kZWorkers;
    float bias_h[COUT / 2];  // this worker's half of the biases
#pragma unroll
    for (int j = 0; j < COUT / 2; ++j) bias_h[j] = worker ? bias[((t >> 7) & 1) * (COUT / 2) + j] : 0.0f;
    if (worker) {
        for (int zz = za - 1; zz <= za + 1 && za < zb; ++zz)
            dhalo_load_plane<CIN>(g, in, x0, y0, zz, Hs + ring_slot(zz) * SLOT);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
        if (za + 2 <= zb) dhalo_load_plane<CIN>(g, in, x0, y0, za + 2, Hs + ring_slot(za + 2) * SLOT);
        asm volatile("cp.async.commit_group;\n" ::: "memory");
    }
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");  // planes za-1 .. za+1 in; za+2 may be in flight
    tc::fence_smem_async();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tslot;
    const uint32_t idesc = tc::idesc_bf16(kTileM, COUT, 0, 0);
    const uint32_t h0 = tc::smem_addr(Hs), b0 = tc::smem_addr(Bs);
    // a worker's cell in a tile of plane z: M row t % 128
    const int64_t cxy = (int64_t)(y0 + (t & 127) / 8) * g.nx + x0 + (t & 7);
    uint32_t uses[2] = {0, 0};
    bool ok = true;
    int n = 0;
    for (int z = za; z < zb && ok; ++z, ++n) {
        const int b = n & 1;
        if (t == kZIssuer) {
            // planes z-1 .. z+1 were copied before the last barrier, and the
            // previous tile of accumulator b (z - 2) was read before it
            const uint64_t db0 = tc::smem_desc(b0, 128, 256);
#pragma unroll
            for (int tap = 0; tap < 27; ++tap) {
                const int dx = tap % 3 - 1, dy = (tap / 3) % 3 - 1, dz = tap / 9 - 1;
                // the start address is the descriptor's low field (16-byte
                // units, smem < 256 KB so no carry): offsets add directly
                const uint64_t da = tc::smem_desc(h0 + ring_slot(z + dz) * SLOT, KG * 16, kHX * 16);
#pragma unroll
                for (int kb = 0; kb < KS; ++kb) {
                    const uint32_t aoff = 2 * kb * KG + (uint32_t)((1 + dy) * kHX + 1 + dx);
                    const uint32_t boff = (uint32_t)((tap * KS + kb) * COUT * 32 / 16);
                    tc::mma_bf16(tmem + b * 32, da + aoff, db0 + boff, idesc, (tap > 0 || kb > 0) ? 1u : 0u);
                }
            }
            tc::mma_commit(&bar[b]);
        }
        ++uses[b];
        bool lost = false;
        if (worker) {
            // tile z - 1 done: its accumulator is final, and the slot of plane
            // z - 2, which only it still read, takes plane z + 3
            if (uses[b ^ 1] > 0) lost = !tc::mbar_wait(&bar[b ^ 1], (uses[b ^ 1] - 1) & 1, err, wait_limit);
            if (!lost) {
                tc::fence_after_sync();
                if (z + 3 <= zb) dhalo_load_plane<CIN>(g, in, x0, y0, z + 3, Hs + ring_slot(z + 3) * SLOT);
                asm volatile("cp.async.commit_group;\n" ::: "memory");
                if (z > za)
                    conv_epilogue<COUT, MODE>(tmem + (b ^ 1) * 32, (int64_t)(z - 1) * g.nx * g.ny + cxy, bias_h,
                                              pre_below, out_pre, out_bf, out_f);
            }
            // plane z + 2 in (tile z + 1 reads it); z + 3 may stay in flight
            if (lost) asm volatile("cp.async.wait_all;\n" ::: "memory");
            else asm volatile("cp.async.wait_group 1;\n" ::: "memory");
            tc::fence_smem_async();
        }
        tc::fence_before_sync();
        if (__syncthreads_or(lost)) {  // plane z + 2 visible; accumulator b^1 read
            ok = false;
            break;
        }
        tc::fence_after_sync();
    }
    if (ok && n > 0) {
        const int b = (n - 1) & 1;
        bool lost = false;
        if (worker) lost = !tc::mbar_wait(&bar[b], (uses[b] - 1) & 1, err, wait_limit);
        if (!__syncthreads_or(lost) && worker) {
            tc::fence_after_sync();
            conv_epilogue<COUT, MODE>(tmem + b * 32, (int64_t)(zb - 1) * g.nx * g.ny + cxy, bias_h, pre_below,
                                      out_pre, out_bf, out_f);
        }
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");  // no copy outlives the block
    if (t == 0) {
        for (int s = 0; s < 2; ++s)
            if (uses[s] > 0) tc::mbar_wait(&bar[s], (uses[s] - 1) & 1, err);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (t < 32) tc::tmem_dealloc(tmem, 64);
}

// Weight gradient dW[tap][ci][co] = sum_c act[c + off(tap)][ci] * grad[c][co]
// over this CTA's cell range, as partials[cta][tap][ci][co] (FP32).
// M rows = (tap-in-group j, ci), TPG = 128/CIN taps per group, G groups;
// K = cells, 32 per stage (2 k-steps); operands MN-major.
template <int CIN, int COUT>
struct WGradShape {
    static constexpr int TPG = kTileM / CIN;
    static constexpr int G = (27 + TPG - 1) / TPG;
    static constexpr int COLS = G * COUT;
    static constexpr int TCOLS = COLS <= 32 ? 32 : (COLS <= 64 ? 64 : (COLS <= 128 ? 128 : 256));
    static constexpr int KC = 32;                                  // cells per stage
    static constexpr int ABLK = 4096;                              // 128 x 16 BF16
    static constexpr int BBLK = COUT * 32;                         // COUT x 16 BF16
    static constexpr int STAGE = G * 2 * ABLK + 2 * BBLK;
    static constexpr int SMEM = 2 * STAGE;
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(kThreads) wgrad_kernel(Grid3 g, const __nv_bfloat16* __restrict__ act,
                                                         const __nv_bfloat16* __restrict__ grad,
                                                         float* __restrict__ partials, int* __restrict__ err,
        uint32_t wait_limit) {
    using WS = WGradShape<CIN, COUT>;
    constexpr int TPG = WS::TPG, G = WS::G, KC = WS::KC;
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ uint64_t bar[2];
    __shared__ uint32_t tslot;
    const int t = threadIdx.x;
    if (t == 0) {
        tc::mbar_init(&bar[0], 1);
        tc::mbar_init(&bar[1], 1);
        tc::mbar_fence_init();
    }
    if (t < 32) tc::tmem_alloc(&tslot, WS::TCOLS);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tslot;
    const uint32_t idesc = tc::idesc_bf16(kTileM, COUT, 1, 1);
    const uint32_t s0 = tc::smem_addr(sm);
    uint32_t uses[2] = {0, 0};
    bool ok = true;

    const int64_t nchunks = (g.V + KC - 1) / KC;
    const int64_t ch0 = nchunks * blockIdx.x / gridDim.x, ch1 = nchunks * (blockIdx.x + 1) / gridDim.x;
    bool first = true;
    for (int64_t ch = ch0; ch < ch1; ++ch) {
        const int s = (int)((ch - ch0) & 1);
        bool lost = uses[s] > 0 && !tc::mbar_wait(&bar[s], (uses[s] - 1) & 1, err, wait_limit);
        if (__syncthreads_or(lost)) {
            ok = false;
            break;
        }
        unsigned char* st = sm + s * WS::STAGE;
        // A: item = (slot = tap slot of 28 or 32, q = ci chunk of 8, k = cell of KC)
        constexpr int NA = G * TPG * (CIN / 8) * KC;
        for (int i = t; i < NA; i += kThreads) {
            const int q = i % (CIN / 8);
            const int k = (i / (CIN / 8)) % KC;
            const int slot = i / ((CIN / 8) * KC);
            const int gi = slot / TPG, j = slot % TPG;
            const int64_t c = ch * KC + k;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (slot < 27 && c < g.V) {
                const int x = (int)(c % g.nx), y = (int)((c / g.nx) % g.ny), z = (int)(c / ((int64_t)g.nx * g.ny));
                v = reinterpret_cast<const uint4*>(act + neighbour(g, x, y, z, slot) * CIN)[q];
            }
            const int m = j * CIN + q * 8;
            const int kk = k % 16;
            *reinterpret_cast<uint4*>(st + (gi * 2 + k / 16) * WS::ABLK + (m / 8) * 128 + (kk / 8) * 2048 +
                                      (kk % 8) * 16) = v;
        }
        // B: item = (q = co chunk of 8, k)
        unsigned char* bst = st + G * 2 * WS::ABLK;
        for (int i = t; i < (COUT / 8) * KC; i += kThreads) {
            const int q = i % (COUT / 8), k = i / (COUT / 8);
            const int64_t c = ch * KC + k;
            uint4 v = make_uint4(0, 0, 0, 0);
            if (c < g.V) v = reinterpret_cast<const uint4*>(grad + c * COUT)[q];
            const int kk = k % 16;
            *reinterpret_cast<uint4*>(bst + (k / 16) * WS::BBLK + q * 128 + (kk / 8) * (COUT / 8) * 128 +
                                      (kk % 8) * 16) = v;
        }
        tc::fence_smem_async();
        tc::fence_before_sync();
        __syncthreads();
        tc::fence_after_sync();
        if (t == 0) {
            const uint32_t sa = s0 + s * WS::STAGE;
#pragma unroll 1
            for (int gi = 0; gi < G; ++gi) {
#pragma unroll
                for (int ks = 0; ks < 2; ++ks) {
                    const uint64_t da = tc::smem_desc(sa + (gi * 2 + ks) * WS::ABLK, 2048, 128);
                    const uint64_t db = tc::smem_desc(sa + G * 2 * WS::ABLK + ks * WS::BBLK, (COUT / 8) * 128, 128);
                    tc::mma_bf16(tmem + gi * COUT, da, db, idesc, (first && ks == 0) ? 0u : 1u);
                }
            }
            tc::mma_commit(&bar[s]);
        }
        first = false;
        ++uses[s];
    }
    if (ok && uses[0] + uses[1] > 0) {
        const int last = (int)(((ch1 - ch0) - 1) & 1);
        const bool lost = !tc::mbar_wait(&bar[last], (uses[last] - 1) & 1, err, wait_limit);
        ok = !__syncthreads_or(lost);
    }
    tc::fence_after_sync();
    if (ok) {
        const int w = t >> 5;
        const int j = t / CIN, ci = t % CIN;
        float* dst = partials + (int64_t)blockIdx.x * 27 * CIN * COUT;
        for (int gi = 0; gi < G; ++gi) {
            float v[COUT];
            if (first) {
#pragma unroll
                for (int co = 0; co < COUT; ++co) v[co] = 0.0f;  // no cells: zero partial
            } else {
#pragma unroll
                for (int c0 = 0; c0 < COUT; c0 += 16)
                    tc::tmem_ld16(tmem + ((uint32_t)(32 * w) << 16) + (uint32_t)(gi * COUT + c0), v + c0);
            }
            const int tap = gi * TPG + j;
            if (tap < 27) {
#pragma unroll
                for (int co = 0; co < COUT; ++co) dst[((int64_t)tap * CIN + ci) * COUT + co] = v[co];
            }
        }
    }
    if (t == 0) {
        for (int s = 0; s < 2; ++s)
            if (uses[s] > 0) tc::mbar_wait(&bar[s], (uses[s] - 1) & 1, err);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (t < 32) tc::tmem_dealloc(tmem, WS::TCOLS);
}

// The weight gradient's per-tile halo: the 10 x 18 x 3 neighbourhood of an
// 8 x 16 x 1 tile as 16-byte units, one block per 8-channel group:
//   unit(kg, hz, hy, hx) at ((kg*3 + hz)*18 + hy)*10 + hx.
constexpr int kHZ = 3;
__host__ __device__ constexpr int whalo_bytes(int cin) { return (cin / 8) * kHX * kHY * kHZ * 16; }

template <int CIN>
__device__ __forceinline__ void whalo_load(const Grid3& g, const __nv_bfloat16* __restrict__ in, int x0, int y0,
                                           int z0, unsigned char* H) {
    constexpr int QU = CIN / 8;
    constexpr int N = QU * kHX * kHY * kHZ;
    for (int i = threadIdx.x; i < N; i += kThreads) {
        const int hx = i % kHX, hy = (i / kHX) % kHY, hz = (i / (kHX * kHY)) % kHZ, kg = i / (kHX * kHY * kHZ);
        const int64_t cell =
            ((int64_t)wrapi(z0 - 1 + hz, g.nz) * g.ny + wrapi(y0 - 1 + hy, g.ny)) * g.nx + wrapi(x0 - 1 + hx, g.nx);
        const uint4* src = reinterpret_cast<const uint4*>(in + cell * CIN) + kg;
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(tc::smem_addr(H + i * 16)), "l"(src));
    }
}

// Weight gradient on 8 x 16 x 1 tiles (nx % 8 == 0, ny % 16 == 0).  Per tile
// the activation halo (above) and the tile's
// output gradient are staged once; then for each group of TPG taps the
// MN-major A operand (rows (tap, ci), K = the tile's 128 cells) is assembled
// from the halo by 16-byte copies -- cell k of the tile is row k of every
// 8-channel plane, so K-groups are 128 bytes apart and channel groups 2 KB --
// and 8 K-steps of MMAs accumulate into the group's TMEM columns.  Two A
// buffers let the copies of one group overlap the MMAs of the previous one.
template <int CIN, int COUT>
struct WGradHalo {
    static constexpr int TPG = kTileM / CIN;
    static constexpr int G = (27 + TPG - 1) / TPG;
    static constexpr int TCOLS = WGradShape<CIN, COUT>::TCOLS;
    static constexpr int HB = whalo_bytes(CIN);
    static constexpr int BB = (COUT / 8) * 2048;  // output-gradient tile
    static constexpr int AB = 16 * 2048;          // one A buffer (128 x 128 BF16)
    static constexpr int SMEM = HB + BB + 2 * AB;
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(kThreads) wgrad_dhalo_kernel(Grid3 g, const __nv_bfloat16* __restrict__ act,
                                                               const __nv_bfloat16* __restrict__ grad,
                                                               float* __restrict__ partials, int* __restrict__ err,
        uint32_t wait_limit) {
    using WH = WGradHalo<CIN, COUT>;
    constexpr int TPG = WH::TPG, G = WH::G, QU = CIN / 8;
    extern __shared__ __align__(1024) unsigned char sm[];
    __shared__ uint64_t bar[2];
    __shared__ uint32_t tslot;
    unsigned char* Hs = sm;
    unsigned char* Bs = sm + WH::HB;
    unsigned char* As = Bs + WH::BB;
    const int t = threadIdx.x;
    if (t == 0) {
        tc::mbar_init(&bar[0], 1);
        tc::mbar_init(&bar[1], 1);
        tc::mbar_fence_init();
    }
    if (t < 32) tc::tmem_alloc(&tslot, WH::TCOLS);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tmem = tslot;
    const uint32_t idesc = tc::idesc_bf16(kTileM, COUT, 1, 1);
    const uint32_t a0 = tc::smem_addr(As), b0 = tc::smem_addr(Bs);
    const int bx = g.nx / 8, by = g.ny / 16;
    const int64_t ntiles = (int64_t)bx * by * g.nz;
    uint32_t uses[2] = {0, 0};
    int kg_run = 0;  // groups issued so far (selects the A buffer)
    int last_b = -1;
    bool ok = true, any = false;
    for (int64_t tile = blockIdx.x; tile < ntiles && ok; tile += gridDim.x) {
        const int x0 = (int)(tile % bx) * 8, y0 = (int)((tile / bx) % by) * 16;
        const int z0 = (int)(tile / ((int64_t)bx * by));
        // the previous tile's MMAs read the gradient tile: let them finish
        bool lost = last_b >= 0 && !tc::mbar_wait(&bar[last_b], (uses[last_b] - 1) & 1, err, wait_limit);
        if (__syncthreads_or(lost)) {
            ok = false;
            break;
        }
        whalo_load<CIN>(g, act, x0, y0, z0, Hs);
        for (int i = t; i < (COUT / 8) * 128; i += kThreads) {
            const int k = i % 128, q = i / 128;
            const int64_t cell = ((int64_t)z0 * g.ny + y0 + k / 8) * g.nx + x0 + k % 8;
            const uint4* src = reinterpret_cast<const uint4*>(grad + cell * COUT) + q;
            asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(tc::smem_addr(Bs + q * 2048 + k * 16)),
                         "l"(src));
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");
        __syncthreads();
        for (int gi = 0; gi < G; ++gi, ++kg_run) {
            const int b = kg_run & 1;
            lost = uses[b] > 0 && !tc::mbar_wait(&bar[b], (uses[b] - 1) & 1, err, wait_limit);
            if (__syncthreads_or(lost)) {
                ok = false;
                break;
            }
            unsigned char* A = As + b * WH::AB;
            for (int i = t; i < TPG * QU * 128; i += kThreads) {
                const int k = i % 128, kg = (i / 128) % QU, j = i / (128 * QU);
                const int tap = gi * TPG + j;
                uint4 v = make_uint4(0, 0, 0, 0);
                if (tap < 27) {
                    const int dx = tap % 3 - 1, dy = (tap / 3) % 3 - 1, dz = tap / 9 - 1;
                    const int hu = ((kg * kHZ + 1 + dz) * kHY + 1 + dy + k / 8) * kHX + 1 + dx + k % 8;
                    v = *reinterpret_cast<const uint4*>(Hs + hu * 16);
                }
                *reinterpret_cast<uint4*>(A + (j * QU + kg) * 2048 + k * 16) = v;
            }
            tc::fence_smem_async();
            tc::fence_before_sync();
            __syncthreads();
            tc::fence_after_sync();
            if (t == 0) {
                const uint64_t da0 = tc::smem_desc(a0 + b * WH::AB, 128, 2048);
                const uint64_t db0 = tc::smem_desc(b0, 128, 2048);
#pragma unroll
                for (int ks = 0; ks < 8; ++ks)
                    tc::mma_bf16(tmem + gi * COUT, da0 + (uint32_t)(ks * 256 / 16), db0 + (uint32_t)(ks * 256 / 16),
                                 idesc, (any || ks > 0) ? 1u : 0u);
                tc::mma_commit(&bar[b]);
            }
            ++uses[b];
            last_b = b;
        }
        any = true;
    }
    if (ok && last_b >= 0) {
        const bool lost = !tc::mbar_wait(&bar[last_b], (uses[last_b] - 1) & 1, err, wait_limit);
        ok = !__syncthreads_or(lost);
    }
    tc::fence_after_sync();
    if (ok) {
        const int w = t >> 5;
        const int j = t / CIN, ci = t % CIN;
        float* dst = partials + (int64_t)blockIdx.x * 27 * CIN * COUT;
        for (int gi = 0; gi < G; ++gi) {
            float v[COUT];
            if (!any) {
#pragma unroll
                for (int co = 0; co < COUT; ++co) v[co] = 0.0f;
            } else {
#pragma unroll
                for (int c0 = 0; c0 < COUT; c0 += 16)
                    tc::tmem_ld16(tmem + ((uint32_t)(32 * w) << 16) + (uint32_t)(gi * COUT + c0), v + c0);
            }
            const int tap = gi * TPG + j;
            if (tap < 27) {
#pragma unroll
                for (int co = 0; co < COUT; ++co) dst[((int64_t)tap * CIN + ci) * COUT + co] = v[co];
            }
        }
    }
    if (t == 0) {
        for (int s = 0; s < 2; ++s)
            if (uses[s] > 0) tc::mbar_wait(&bar[s], (uses[s] - 1) & 1, err);
    }
    tc::fence_before_sync();
    __syncthreads();
    if (t < 32) tc::tmem_dealloc(tmem, WH::TCOLS);
}

// out[j] = sum over p < P of partials[p * n + j] in a fixed order: a block
// takes 32 consecutive j; its warp s sums the partials p = s, s + 8, ... in
// increasing p, then the 8 slice sums are added in increasing s.  (One
// thread per j summing all P serially left most SMs idle.)  Launch with
// kFoldThreads threads and ceil(n / 32) blocks.
constexpr int kFoldThreads = 256;
__global__ void __launch_bounds__(kFoldThreads) sum_partials_kernel(const float* __restrict__ partials, int P, int n,
                                                                     float* __restrict__ out) {
    __shared__ float slice[kFoldThreads / 32][32];
    const int lane = threadIdx.x & 31, s = threadIdx.x >> 5;
    const int j = blockIdx.x * 32 + lane;
    float acc = 0.0f;
    if (j < n)
        for (int p = s; p < P; p += kFoldThreads / 32) acc += partials[(int64_t)p * n + j];
    slice[s][lane] = acc;
    __syncthreads();
    if (s == 0 && j < n) {
        float t = slice[0][lane];
#pragma unroll
        for (int k = 1; k < kFoldThreads / 32; ++k) t += slice[k][lane];
        out[j] = t;
    }
}

// Bias gradient partials: per block, sum over its cells of grad[c][co].
template <int C>
__global__ void bias_grad_kernel(const __nv_bfloat16* __restrict__ grad, int64_t V, float* __restrict__ partials) {
    __shared__ float sh[kThreads / 32][C];
    float acc[C];
#pragma unroll
    for (int j = 0; j < C; ++j) acc[j] = 0.0f;
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < V; c += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int j = 0; j < C; ++j) acc[j] += __bfloat162float(grad[c * C + j]);
    }
#pragma unroll
    for (int j = 0; j < C; ++j) {
        float v = acc[j];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5][j] = v;
    }
    __syncthreads();
    if (threadIdx.x < C) {
        float v = 0.0f;
        for (int w = 0; w < kThreads / 32; ++w) v += sh[w][threadIdx.x];
        partials[(int64_t)blockIdx.x * C + threadIdx.x] = v;
    }
}

// Fwd and backward-data B images of one layer from the FP32 master weights
// W[27][CIN][COUT] (padding rows/columns are zero in the master copy).
template <int CIN, int COUT>
__global__ void pack_kernel(const float* __restrict__ W, __nv_bfloat16* __restrict__ fwd,
                            __nv_bfloat16* __restrict__ bwd) {
    const int n = 27 * CIN * COUT;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int co = i % COUT, ci = (i / COUT) % CIN, tap = i / (CIN * COUT);
        const __nv_bfloat16 v = __float2bfloat16(W[i]);
        {  // forward: B[n = co][k = ci] of k-step (tap, ci/16)
            const int s = tap * (CIN / 16) + ci / 16, k = ci % 16;
            fwd[(s * COUT * 32 + tc::kmajor_off(co, k, 128, 256)) / 2] = v;
        }
        if (bwd) {  // backward data: tap' = 26 - tap, B[n = ci][k = co]
            const int tp = 26 - tap;
            const int s = tp * (COUT / 16) + co / 16, k = co % 16;
            bwd[(s * CIN * 32 + tc::kmajor_off(ci, k, 128, 256)) / 2] = v;
        }
    }
}

// Adam on the flat FP32 parameter vector.
__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ grad, float* __restrict__ m,
                            float* __restrict__ v, const float* __restrict__ mask, int n, float lr, float b1,
                            float b2, float eps, float bc1, float bc2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = grad[i] * mask[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= mask[i] * lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    }
}

// Standard normal variate from a counter (splitmix64 of key and index,
// Box-Muller), for training-input noise.
__device__ __forceinline__ float hash_normal(uint64_t key, uint64_t i) {
    auto mix = [](uint64_t z) {
        z += 0x9e3779b97f4a7c15ull;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return z ^ (z >> 31);
    };
    const uint64_t h = mix(key ^ mix(i));
    const float u1 = ((float)(h >> 40) + 0.5f) * 0x1.0p-24f, u2 = (float)((h >> 16) & 0xFFFFFF) * 0x1.0p-24f;
    return sqrtf(-2.0f * logf(u1)) * cospif(2.0f * u2);
}

// Network input from 9 FP32 channel blocks (rho, u, Q; [9][V]):
// act0[c][j] = (x_j - shift_j) * inv_scale_j (+ noise_std N(0,1) when
// training with input noise) for j < 9, 0 for j in 9..15.
__global__ void features_kernel(const float* __restrict__ rho, const float* __restrict__ u3,
                                const float* __restrict__ q5, int64_t V, const float* __restrict__ shift,
                                const float* __restrict__ inv_scale, __nv_bfloat16* __restrict__ act0,
                                float noise_std, uint64_t noise_key) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < V; c += (int64_t)gridDim.x * blockDim.x) {
        __align__(16) __nv_bfloat16 v[16];
        float x[9];
        x[0] = rho[c];
#pragma unroll
        for (int k = 0; k < 3; ++k) x[1 + k] = u3[k * V + c];
#pragma unroll
        for (int k = 0; k < 5; ++k) x[4 + k] = q5[k * V + c];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            float f = 0.0f;
            if (j < 9) {
                f = (x[j] - shift[j]) * inv_scale[j];
                if (noise_std > 0.0f) f += noise_std * hash_normal(noise_key, (uint64_t)c * 16 + j);
            }
            v[j] = __float2bfloat16(f);
        }
        reinterpret_cast<uint4*>(act0 + c * 16)[0] = reinterpret_cast<const uint4*>(v)[0];
        reinterpret_cast<uint4*>(act0 + c * 16)[1] = reinterpret_cast<const uint4*>(v)[1];
    }
}

// Mean-squared error of the 8 outputs against the raw targets [8][V]
// normalised by inv_scale, its gradient gout[c][16] (BF16, channels 8..15
// zero) and per-block partial sums of the squared error.
__global__ void __launch_bounds__(kThreads) loss_kernel(const float* __restrict__ out, const float* __restrict__ tgt,
                                                        const float* __restrict__ inv_scale, int64_t V,
                                                        __nv_bfloat16* __restrict__ gout,
                                                        double* __restrict__ partials) {
    __shared__ double sh[kThreads / 32];
    double acc = 0.0;
    const float gscale = 2.0f / (8.0f * (float)V);
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < V; c += (int64_t)gridDim.x * blockDim.x) {
        __align__(16) __nv_bfloat16 gv[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            float gj = 0.0f;
            if (j < 8) {
                const float d = out[c * 16 + j] - tgt[j * V + c] * inv_scale[j];
                acc += (double)d * d;
                gj = gscale * d;
            }
            gv[j] = __float2bfloat16(gj);
        }
        reinterpret_cast<uint4*>(gout + c * 16)[0] = reinterpret_cast<const uint4*>(gv)[0];
        reinterpret_cast<uint4*>(gout + c * 16)[1] = reinterpret_cast<const uint4*>(gv)[1];
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double v = 0.0;
        for (int w = 0; w < kThreads / 32; ++w) v += sh[w];
        partials[blockIdx.x] = v;
    }
}

// Correction of a coarse state after its step: Q_k += gain out[c][k] s_k
// (k < 5), u_d += gain out[c][5+d] s_{5+d}.
__global__ void apply_kernel(const float* __restrict__ out, const float* __restrict__ out_scale, int64_t V,
                             float gain, float* __restrict__ u3, float* __restrict__ q5) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < V; c += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k < 5; ++k) q5[k * V + c] += gain * out[c * 16 + k] * out_scale[k];
#pragma unroll
        for (int d = 0; d < 3; ++d) u3[d * V + c] += gain * out[c * 16 + 5 + d] * out_scale[5 + d];
    }
}

// Box filter of a fine state (factor f per axis) onto the coarse grid:
// rho_c = <rho>, u_c = <rho u> / rho_c, Q_c = <Q>; out [9][Vc].
__global__ void filter_kernel(const float* __restrict__ rho, const float* __restrict__ u3,
                              const float* __restrict__ q5, int nx, int ny, int nz, int f,
                              float* __restrict__ out) {
    const int cx = nx / f, cy = ny / f, cz = nz / f;
    const int64_t Vc = (int64_t)cx * cy * cz, V = (int64_t)nx * ny * nz;
    const double inv = 1.0 / ((double)f * f * f);
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < Vc; c += (int64_t)gridDim.x * blockDim.x) {
        const int X = (int)(c % cx), Y = (int)((c / cx) % cy), Z = (int)(c / ((int64_t)cx * cy));
        double r = 0, m[3] = {0, 0, 0}, q[5] = {0, 0, 0, 0, 0};
        for (int dz = 0; dz < f; ++dz)
            for (int dy = 0; dy < f; ++dy)
                for (int dx = 0; dx < f; ++dx) {
                    const int64_t i = ((int64_t)(Z * f + dz) * ny + (Y * f + dy)) * nx + (X * f + dx);
                    const double ri = rho[i];
                    r += ri;
#pragma unroll
                    for (int d = 0; d < 3; ++d) m[d] += ri * u3[d * V + i];
#pragma unroll
                    for (int k = 0; k < 5; ++k) q[k] += q5[k * V + i];
                }
        out[c] = (float)(r * inv);
#pragma unroll
        for (int d = 0; d < 3; ++d) out[(1 + d) * Vc + c] = (float)(m[d] / r);
#pragma unroll
        for (int k = 0; k < 5; ++k) out[(4 + k) * Vc + c] = (float)(q[k] * inv);
    }
}

// Per-block sums and sums of squares of nc channel blocks [nc][V] (or a
// difference a - b when b is given): partials[(blk * nc + j) * 2 + {0,1}].
__global__ void __launch_bounds__(kThreads) moments_kernel(const float* __restrict__ a, const float* __restrict__ b,
                                                           int nc, int64_t V, double* __restrict__ partials) {
    __shared__ double sh[2][kThreads / 32];
    for (int j = 0; j < nc; ++j) {
        double s1 = 0.0, s2 = 0.0;
        for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < V;
             c += (int64_t)gridDim.x * blockDim.x) {
            const double x = (double)a[j * V + c] - (b ? (double)b[j * V + c] : 0.0);
            s1 += x;
            s2 += x * x;
        }
        for (int o = 16; o > 0; o >>= 1) {
            s1 += __shfl_xor_sync(0xffffffffu, s1, o);
            s2 += __shfl_xor_sync(0xffffffffu, s2, o);
        }
        if ((threadIdx.x & 31) == 0) {
            sh[0][threadIdx.x >> 5] = s1;
            sh[1][threadIdx.x >> 5] = s2;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double v1 = 0.0, v2 = 0.0;
            for (int w = 0; w < kThreads / 32; ++w) {
                v1 += sh[0][w];
                v2 += sh[1][w];
            }
            partials[((int64_t)blockIdx.x * nc + j) * 2] = v1;
            partials[((int64_t)blockIdx.x * nc + j) * 2 + 1] = v2;
        }
        __syncthreads();
    }
}

// Raw training target [8][V]: next - pred, Q components then u.
__global__ void target_kernel(const float* __restrict__ next9, const float* __restrict__ pu3,
                              const float* __restrict__ pq5, int64_t V, float* __restrict__ tgt) {
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < V; c += (int64_t)gridDim.x * blockDim.x) {
#pragma unroll
        for (int k = 0; k < 5; ++k) tgt[k * V + c] = next9[(4 + k) * V + c] - pq5[k * V + c];
#pragma unroll
        for (int d = 0; d < 3; ++d) tgt[(5 + d) * V + c] = next9[(1 + d) * V + c] - pu3[d * V + c];
    }
}

}  // namespace cl
}  // namespace lbman
