// kernels_impl.cuh -- launcher bodies, instantiated per precision by
// kernels_f64.cu / kernels_f32.cu.
#pragma once

#include "fused.cuh"
#include "init.cuh"
#include "qsplit.cuh"
#include "qpair.cuh"
#include "launch.h"
#include "reduce.cuh"
#include "tiles.h"

#include <algorithm>
#include <atomic>
#include <utility>

namespace lbman {
namespace impl {

inline unsigned blocks_for(int64_t n, int threads) { return (unsigned)((n + threads - 1) / threads); }

inline dim3 qgrid(const SimParams& P, int tcx, int tcy, int zc) {
    return dim3((unsigned)((P.nx + tcx - 1) / tcx), (unsigned)((P.ny + tcy - 1) / tcy),
                (unsigned)((P.zhi - P.zlo + zc - 1) / zc));
}

constexpr size_t kMaxSmem = 227 * 1024;

// Calls f(Tile<...>{}) for the compiled tile shape (tcx, tcy); tiles whose
// staging does not fit in one block's shared memory for this precision are
// not instantiated.  Returns cudaErrorInvalidValue for any other shape.
template <class R, class F>
cudaError_t with_tile(int tcx, int tcy, F&& f) {
#define LBMAN_TILE(X, Y)                                                   \
    if (tcx == X && tcy == Y) {                                            \
        if constexpr (Tile<X, Y>::template smem_bytes<R>() <= kMaxSmem)    \
            return f(Tile<X, Y>{});                                        \
        else                                                               \
            return cudaErrorInvalidValue;                                  \
    }
    LBMAN_TILES(LBMAN_TILE)
#undef LBMAN_TILE
    return cudaErrorInvalidValue;
}

// Calls f(PairTile<...>{}) for a compiled pair tile (FP32 compute only);
// cudaErrorInvalidValue for any other shape or precision.
template <class R, class F>
cudaError_t with_pair_tile(int tcx, int tcy, F&& f) {
    if constexpr (sizeof(R) == 4) {
#define LBMAN_TILE(X, Y)                                                       \
    if (tcx == X && tcy == Y) {                                                \
        if constexpr (PairTile<X, Y>::template smem_bytes<R>() <= kMaxSmem)    \
            return f(PairTile<X, Y>{});                                        \
        else                                                                   \
            return cudaErrorInvalidValue;                                      \
    }
        LBMAN_PAIR_TILES(LBMAN_TILE)
#undef LBMAN_TILE
    }
    return cudaErrorInvalidValue;
}

// with_tile or with_pair_tile, as the shape says
template <class R, class F>
cudaError_t with_qtile(const QTile& T, F&& f) {
    return T.pair ? with_pair_tile<R>(T.tcx, T.tcy, f) : with_tile<R>(T.tcx, T.tcy, f);
}

template <class R>
size_t qforce_smem(const QTile& T) {
    size_t b = 0;
    with_qtile<R>(T, [&](auto tl) {
        b = decltype(tl)::template smem_bytes<R>();
        return cudaSuccess;
    });
    return b;
}

template <class R>
int qforce_threads(const QTile& T) {
    int n = 0;
    with_qtile<R>(T, [&](auto tl) {
        n = decltype(tl)::NT;
        return cudaSuccess;
    });
    return n;
}

// Resident blocks per SM that the SM's shared memory (1 KB reserved per
// block), registers and thread limit admit for a kernel at this shape.
template <auto Kern>
int fit_blocks(int threads, size_t smem) {
    int dev = 0, smem_sm = 0, regs_sm = 0, threads_sm = 0;
    cudaFuncAttributes fa{};
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&threads_sm, cudaDevAttrMaxThreadsPerMultiProcessor, dev) != cudaSuccess ||
        cudaFuncGetAttributes(&fa, Kern) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    int n = (int)((size_t)smem_sm / (smem + fa.sharedSizeBytes + 1024));
    n = std::min(n, regs_sm / std::max(1, fa.numRegs * threads));
    n = std::min(n, threads_sm / threads);
    return std::max(1, n);
}

// Resident blocks per SM of one kernel instantiation at its launch shape
// (computed once; the dynamic shared-memory limit is raised by prepare()).
// The occupancy query and the count from the SM's resources are both taken:
// the query has answered 1 for kernels that run two blocks per SM here.
template <auto Kern>
int resident_blocks(int threads, size_t smem) {
    static std::atomic<int> cached{0};
    int n = cached.load(std::memory_order_relaxed);
    if (n == 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, Kern, threads, smem) != cudaSuccess || n < 1) {
            cudaGetLastError();
            n = 1;
        }
        n = std::max(n, fit_blocks<Kern>(threads, smem));
        cached.store(n, std::memory_order_relaxed);
    }
    return n;
}

// Grid of a z-marching launch: fixed z chunks (zc > 0), or for the balanced
// schedule (zc <= 0) max(1, -zc) waves of resident blocks sharing the
// (column, plane) units equally.
template <class TL, auto Kern>
dim3 march_grid(const SimParams& P, const LaunchShape& S, size_t smem) {
    if (S.tile.zc > 0) return qgrid(P, TL::TCX, TL::TCY, S.tile.zc);
    const int64_t units = (int64_t)((P.nx + TL::TCX - 1) / TL::TCX) * ((P.ny + TL::TCY - 1) / TL::TCY) * (P.zhi - P.zlo);
    const int64_t waves = std::max(1, -S.tile.zc);
    const int64_t grid = waves * resident_blocks<Kern>(TL::NT, smem) * S.num_sms;
    return dim3((unsigned)std::max<int64_t>(1, std::min(units, grid)));
}

// The pair kernel stages 16-byte chunks: nx a multiple of 4 and 16-byte
// aligned fields (every field offset k V is then a multiple of 4 floats).
inline bool pair_ok(const SimParams& P, const void* qin, const void* uin) {
    return (P.nx & 3) == 0 && ((reinterpret_cast<uintptr_t>(qin) | reinterpret_cast<uintptr_t>(uin)) & 15) == 0;
}

template <class R>
cudaError_t qforce(const SimParams& P, const LaunchShape& S, const void* qin, const void* uin, void* qout,
                   void* Fout, cudaStream_t st) {
    if (S.tile.pair) {
        if constexpr (sizeof(R) == 4) {
            if (!pair_ok(P, qin, uin)) return cudaErrorInvalidValue;
            return with_pair_tile<R>(S.tile.tcx, S.tile.tcy, [&](auto tl) {
                using TL = decltype(tl);
                const size_t smem = TL::template smem_bytes<R>();
                if (P.upwind) {
                    constexpr auto K = qpair_kernel<TL, true>;
                    K<<<march_grid<TL, K>(P, S, smem), TL::NT, smem, st>>>(P, S.tile.zc, (const float*)qin,
                                                                           (const float*)uin, (float*)qout,
                                                                           (float*)Fout);
                } else {
                    constexpr auto K = qpair_kernel<TL, false>;
                    K<<<march_grid<TL, K>(P, S, smem), TL::NT, smem, st>>>(P, S.tile.zc, (const float*)qin,
                                                                           (const float*)uin, (float*)qout,
                                                                           (float*)Fout);
                }
                return cudaGetLastError();
            });
        }
        return cudaErrorInvalidValue;
    }
    return with_tile<R>(S.tile.tcx, S.tile.tcy, [&](auto tl) {
        using TL = decltype(tl);
        const size_t smem = TL::template smem_bytes<R>();
        if (P.upwind) {
            constexpr auto K = qforce_kernel<TL, R, true>;
            K<<<march_grid<TL, K>(P, S, smem), TL::NT, smem, st>>>(P, S.tile.zc, (const R*)qin, (const R*)uin,
                                                                   (R*)qout, (R*)Fout);
        } else {
            constexpr auto K = qforce_kernel<TL, R, false>;
            K<<<march_grid<TL, K>(P, S, smem), TL::NT, smem, st>>>(P, S.tile.zc, (const R*)qin, (const R*)uin,
                                                                   (R*)qout, (R*)Fout);
        }
        return cudaGetLastError();
    });
}

template <class R, class S, bool DEV>
cudaError_t fused(const SimParams& P, const LaunchShape& L, bool first, const void* qin, const void* uin,
                  void* qout, void* uout, const void* fin, void* fout, void* rho, void* Fout, bool wr,
                  cudaStream_t st) {
    return with_tile<R>(L.tile.tcx, L.tile.tcy, [&](auto tl) {
        using TL = decltype(tl);
        const size_t smem = TL::template smem_bytes<R>();
        auto launch = [&](auto kern, dim3 g) {
            kern<<<g, TL::NT, smem, st>>>(P, L.tile.zc, first ? 1 : 0, (const R*)qin, (const R*)uin, (R*)qout,
                                          (R*)uout, (const S*)fin, (S*)fout, (R*)rho, (R*)Fout, wr ? 1 : 0);
        };
        if (P.upwind) {
            constexpr auto K = fused_kernel<TL, R, S, DEV, true>;
            launch(K, march_grid<TL, K>(P, L, smem));
        } else {
            constexpr auto K = fused_kernel<TL, R, S, DEV, false>;
            launch(K, march_grid<TL, K>(P, L, smem));
        }
        return cudaGetLastError();
    });
}

// Blocks of the Q+force (or fused) launch for this shape.
template <class R, class S, bool DEV>
int march_blocks(const SimParams& P, const LaunchShape& L, bool fused_org) {
    int n = 0;
    if (L.tile.pair) {
        if constexpr (sizeof(R) == 4) {
            with_pair_tile<R>(L.tile.tcx, L.tile.tcy, [&](auto tl) {
                using TL = decltype(tl);
                const size_t smem = TL::template smem_bytes<R>();
                const dim3 g = P.upwind ? march_grid<TL, qpair_kernel<TL, true>>(P, L, smem)
                                        : march_grid<TL, qpair_kernel<TL, false>>(P, L, smem);
                n = (int)(g.x * g.y * g.z);
                return cudaSuccess;
            });
        }
        return n;
    }
    with_tile<R>(L.tile.tcx, L.tile.tcy, [&](auto tl) {
        using TL = decltype(tl);
        const size_t smem = TL::template smem_bytes<R>();
        dim3 g;
        if (fused_org)
            g = P.upwind ? march_grid<TL, fused_kernel<TL, R, S, DEV, true>>(P, L, smem)
                         : march_grid<TL, fused_kernel<TL, R, S, DEV, false>>(P, L, smem);
        else
            g = P.upwind ? march_grid<TL, qforce_kernel<TL, R, true>>(P, L, smem)
                         : march_grid<TL, qforce_kernel<TL, R, false>>(P, L, smem);
        n = (int)(g.x * g.y * g.z);
        return cudaSuccess;
    });
    return n;
}

template <class R, class S, bool DEV>
cudaError_t lbm(const SimParams& P, bool first, bool wr, const void* fin, void* fout, const void* F,
                void* rho, void* uout, cudaStream_t st) {
    const FastDiv dnx = make_fastdiv((uint32_t)P.nx), dnxy = make_fastdiv((uint32_t)P.nxy);
    const unsigned nb = blocks_for(P.V, 256);
    auto launch = [&](auto kern) {
        kern<<<nb, 256, 0, st>>>(P, dnx, dnxy, first ? 1 : 0, (const S*)fin, (S*)fout, (const R*)F, (R*)rho,
                                 (R*)uout, wr ? 1 : 0);
    };
    const bool walls = !(P.uper[0] && P.uper[2] && P.uper[4]);
    // 32-bit index arithmetic where every population offset fits in an int.
    // Measured on B200 it pays for FP16 storage (5-7%), FP64 (2-4%) and the
    // walled FP32 form (1%), and costs the periodic FP32 form 1-2%.
    if (!(sizeof(S) == 4 && !walls)) {
        if (15 * P.V < ((int64_t)1 << 31)) {
            if (walls) launch(lbm_kernel<R, S, DEV, true, int>);
            else launch(lbm_kernel<R, S, DEV, false, int>);
            return cudaGetLastError();
        }
    }
    if (walls) launch(lbm_kernel<R, S, DEV, true, int64_t>);
    else launch(lbm_kernel<R, S, DEV, false, int64_t>);
    return cudaGetLastError();
}

// One in-place (AA) LBM step: even (PRE -> SWAP) or odd (SWAP -> PRE).
template <class R, class S, bool DEV>
cudaError_t lbm_aa(const SimParams& P, bool odd, bool wr, void* f, const void* F, void* rho, void* uout,
                   cudaStream_t st) {
    const FastDiv dnx = make_fastdiv((uint32_t)P.nx), dnxy = make_fastdiv((uint32_t)P.nxy);
    const unsigned nb = blocks_for(P.c1 - P.c0, 256);
    auto launch = [&](auto kern) {
        kern<<<nb, 256, 0, st>>>(P, dnx, dnxy, (S*)f, (const R*)F, (R*)rho, (R*)uout, wr ? 1 : 0);
    };
    // walled axes (a velocity axis is periodic on both faces or on neither):
    // none, x only (slit), x and y (channel), or any
    const int wm = (P.uper[0] ? 0 : 1) | (P.uper[2] ? 0 : 2) | (P.uper[4] ? 0 : 4);
    const bool i32 = 15 * P.V < ((int64_t)1 << 31);
    // FP16 storage, velocity axes all periodic, nx even: two cells per thread
    // (c0, c1 and V even, so every cell pair's slots are one aligned word)
    if constexpr (sizeof(S) == 2 && sizeof(R) == 4) {
        if (wm == 0 && P.nx % 2 == 0 && (reinterpret_cast<uintptr_t>(f) & 3) == 0) {
            const unsigned nb2 = blocks_for((P.c1 - P.c0) / 2, 256);
            if (odd) {
                auto k = i32 ? lbm_aa_odd_h2_kernel<DEV, int> : lbm_aa_odd_h2_kernel<DEV, int64_t>;
                k<<<nb2, 256, 0, st>>>(P, dnx, dnxy, (S*)f, (const R*)F, (R*)rho, (R*)uout, wr ? 1 : 0);
            } else {
                auto k = i32 ? lbm_aa_even_h2_kernel<DEV, int> : lbm_aa_even_h2_kernel<DEV, int64_t>;
                k<<<nb2, 256, 0, st>>>(P, (S*)f, (const R*)F, (R*)rho, (R*)uout, wr ? 1 : 0);
            }
            return cudaGetLastError();
        }
    }
#define LBMAN_AA(W, I)                                                        \
    do {                                                                      \
        if (odd) launch(lbm_aa_odd_kernel<R, S, DEV, W, I>);                  \
        else launch(lbm_aa_even_kernel<R, S, DEV, W, I>);                     \
    } while (0)
#define LBMAN_AA_I(W)                                                         \
    do {                                                                      \
        if (i32) LBMAN_AA(W, int);                                            \
        else LBMAN_AA(W, int64_t);                                            \
    } while (0)
    if (wm == 0) LBMAN_AA_I(0);
    else if (wm == 1) LBMAN_AA_I(1);
    else if ((wm & ~3) == 0) LBMAN_AA_I(3);
    else LBMAN_AA_I(7);
#undef LBMAN_AA_I
#undef LBMAN_AA
    return cudaGetLastError();
}

template <class R, class S, bool DEV>
cudaError_t aa_pop_out(const SimParams& P, const void* f, const void* rho, double* dst, int dir, cudaStream_t st) {
    const FastDiv dnx = make_fastdiv((uint32_t)P.nx), dnxy = make_fastdiv((uint32_t)P.nxy);
    aa_pop_out_kernel<R, S, DEV><<<blocks_for(P.V, 256), 256, 0, st>>>(P, dnx, dnxy, (const S*)f, (const R*)rho, dst,
                                                                      dir);
    return cudaGetLastError();
}

template <class S>
cudaError_t halo_merge(const SimParams& P, void* f, const void* stage, int face, cudaStream_t st) {
    halo_merge_kernel<S><<<blocks_for(P.nxy, 256), 256, 0, st>>>(P, (S*)f, (const S*)stage, face);
    return cudaGetLastError();
}

template <class S>
cudaError_t swap_pairs(const SimParams& P, void* f, cudaStream_t st) {
    swap_pairs_kernel<S><<<blocks_for(P.V, 256), 256, 0, st>>>(P.V, (S*)f);
    return cudaGetLastError();
}

template <class R, class S>
cudaError_t stream_only(const SimParams& P, const void* fin, void* fout, const void* rho, cudaStream_t st) {
    const FastDiv dnx = make_fastdiv((uint32_t)P.nx), dnxy = make_fastdiv((uint32_t)P.nxy);
    stream_only_kernel<R, S><<<blocks_for(P.V, 256), 256, 0, st>>>(P, dnx, dnxy, (const S*)fin, (S*)fout,
                                                                   (const R*)rho);
    return cudaGetLastError();
}

template <class R, class S, bool DEV>
cudaError_t feq_init(const SimParams& P, const void* rho, const void* u, void* f, cudaStream_t st) {
    feq_init_kernel<R, S, DEV><<<blocks_for(P.V, 256), 256, 0, st>>>(P, (const R*)rho, (const R*)u, (S*)f);
    return cudaGetLastError();
}

__device__ __forceinline__ void to_s(double v, double* d) { *d = v; }
__device__ __forceinline__ void to_s(double v, float* d) { *d = (float)v; }
__device__ __forceinline__ void to_s(double v, __half* d) { *d = __double2half(v); }
__device__ __forceinline__ double from_s(const double* s) { return *s; }
__device__ __forceinline__ double from_s(const float* s) { return (double)*s; }
__device__ __forceinline__ double from_s(const __half* s) { return (double)__half2float(*s); }

template <class T>
__global__ void to_storage_kernel(const double* __restrict__ src, T* __restrict__ dst, int64_t n, double off) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) to_s(src[i] - off, dst + i);
}
template <class T>
__global__ void from_storage_kernel(const T* __restrict__ src, double* __restrict__ dst, int64_t n, double off) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) dst[i] = from_s(src + i) + off;
}

// Populations of direction dir over the cells [c0, c1): host f_i <-> stored
// value (deviation form subtracts w_i rho0); src / dst hold whole-allocation
// arrays.
template <class S, bool DEV>
cudaError_t pop_in(const SimParams& P, const double* src, void* dst, int dir, cudaStream_t st) {
    const double off = DEV ? w_<double>(dir) * P.kDensity : 0.0;
    to_storage_kernel<S><<<blocks_for(P.c1 - P.c0, 256), 256, 0, st>>>(src + P.c0, (S*)dst + (int64_t)dir * P.V + P.c0,
                                                                       P.c1 - P.c0, off);
    return cudaGetLastError();
}
template <class S, bool DEV>
cudaError_t pop_out(const SimParams& P, const void* src, double* dst, int dir, cudaStream_t st) {
    const double off = DEV ? w_<double>(dir) * P.kDensity : 0.0;
    from_storage_kernel<S><<<blocks_for(P.c1 - P.c0, 256), 256, 0, st>>>((const S*)src + (int64_t)dir * P.V + P.c0,
                                                                         dst + P.c0, P.c1 - P.c0, off);
    return cudaGetLastError();
}
template <class R>
cudaError_t real_in(const double* src, void* dst, int64_t n, cudaStream_t st) {
    to_storage_kernel<R><<<blocks_for(n, 256), 256, 0, st>>>(src, (R*)dst, n, 0.0);
    return cudaGetLastError();
}
template <class R>
cudaError_t real_out(const void* src, double* dst, int64_t n, cudaStream_t st) {
    from_storage_kernel<R><<<blocks_for(n, 256), 256, 0, st>>>((const R*)src, dst, n, 0.0);
    return cudaGetLastError();
}

template <class R>
cudaError_t flow_reduce(const SimParams& P, const void* rho, const void* u, void* upast, double* partials, int G,
                        cudaStream_t st) {
    flow_reduce_kernel<R><<<G, kRedThreads, 0, st>>>(P, (const R*)rho, (const R*)u, (R*)upast, partials);
    return cudaGetLastError();
}
template <class R>
cudaError_t energy_reduce(const SimParams& P, const void* q, double* partials, int G, cudaStream_t st) {
    energy_reduce_kernel<R><<<G, kRedThreads, 0, st>>>(P, (const R*)q, partials);
    return cudaGetLastError();
}
template <class R>
cudaError_t director(const SimParams& P, const void* q, void* order, void* dir, int G, cudaStream_t st) {
    director_kernel<R><<<G, kRedThreads, 0, st>>>(P, (const R*)q, (R*)order, (R*)dir);
    return cudaGetLastError();
}
template <class R>
cudaError_t defect_flags(const SimParams& P, const void* dir, uint8_t* flags, int G, cudaStream_t st) {
    defect_flags_kernel<R><<<G, kRedThreads, 0, st>>>(P, (const R*)dir, flags);
    return cudaGetLastError();
}

template <class R>
cudaError_t defect_count(const SimParams& P, const void* dir, double* partials, int G, cudaStream_t st) {
    defect_count_kernel<R><<<G, kRedThreads, 0, st>>>(P, (const R*)dir, partials);
    return cudaGetLastError();
}

template <class R>
cudaError_t seeded_init(const SimParams& P, uint64_t seed, double S0, double sigma, void* rho, void* u, void* q,
                        void* F, cudaStream_t st) {
    const uint64_t key = splitmix64(seed ^ 0x5851f42d4c957f2dULL);
    seeded_init_kernel<R><<<blocks_for(P.c1 - P.c0, 256), 256, 0, st>>>(P, key, S0, sigma, (R*)rho, (R*)u, (R*)q, (R*)F);
    return cudaGetLastError();
}

template <class R>
cudaError_t qsetup(const SimParams& P, const void* qin, const void* uin, void* qout, void* sig, void* tau, void* F,
                   cudaStream_t st) {
    const unsigned nb = blocks_for(P.V, 128);
    if (P.upwind)
        qsetup_kernel<R, true><<<nb, 128, 0, st>>>(P, (const R*)qin, (const R*)uin, (R*)qout, (R*)sig, (R*)tau,
                                                   (R*)F);
    else
        qsetup_kernel<R, false><<<nb, 128, 0, st>>>(P, (const R*)qin, (const R*)uin, (R*)qout, (R*)sig, (R*)tau,
                                                    (R*)F);
    return cudaGetLastError();
}

template <class R>
cudaError_t active_force(const SimParams& P, const void* q, const void* sig, const void* tau, const void* u, void* F,
                         cudaStream_t st) {
    active_force_kernel<R><<<blocks_for(P.V, 128), 128, 0, st>>>(P, (const R*)q, (const R*)sig, (const R*)tau,
                                                                 (const R*)u, (R*)F);
    return cudaGetLastError();
}

template <class R, class S, bool DEV>
cudaError_t prepare(size_t max_smem) {
    const int b = (int)max_smem;
    cudaError_t e = cudaSuccess;
    auto attr = [&](auto kern) {
        if (e == cudaSuccess) e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    };
    for (const auto& xy : kTileList) {
        const int x = xy[0], y = xy[1];
        with_tile<R>(x, y, [&](auto tl) {
            using TL = decltype(tl);
            attr(qforce_kernel<TL, R, true>);
            attr(qforce_kernel<TL, R, false>);
            attr(fused_kernel<TL, R, S, DEV, true>);
            attr(fused_kernel<TL, R, S, DEV, false>);
            return cudaSuccess;
        });
    }
    if constexpr (sizeof(R) == 4) {
        for (const auto& xy : kPairTileList) {
            with_pair_tile<R>(xy[0], xy[1], [&](auto tl) {
                using TL = decltype(tl);
                attr(qpair_kernel<TL, true>);
                attr(qpair_kernel<TL, false>);
                return cudaSuccess;
            });
        }
    }
    return e;
}

}  // namespace impl
}  // namespace lbman

// Defines the launch_*_SUF functions of launch.h for compute type R,
// population storage S and deviation flag DEV.
#define LBMAN_DEFINE_LAUNCHERS(SUF, R, S, DEV)                                                          \
    namespace lbman {                                                                                   \
    cudaError_t launch_qforce_##SUF(const SimParams& P, const LaunchShape& L, const void* qin,          \
                                    const void* uin, void* qout, void* Fout, cudaStream_t st) {        \
        return impl::qforce<R>(P, L, qin, uin, qout, Fout, st);                                         \
    }                                                                                                   \
    cudaError_t launch_fused_##SUF(const SimParams& P, const LaunchShape& L, bool first,                \
                                   const void* qin, const void* uin, void* qout, void* uout,           \
                                   const void* fin, void* fout, void* rho, void* Fout, bool wr,        \
                                   cudaStream_t st) {                                                  \
        return impl::fused<R, S, DEV>(P, L, first, qin, uin, qout, uout, fin, fout, rho, Fout, wr, st); \
    }                                                                                                   \
    cudaError_t launch_lbm_##SUF(const SimParams& P, bool first, bool wr, const void* fin, void* fout,  \
                                 const void* F, void* rho, void* uout, cudaStream_t st) {              \
        return impl::lbm<R, S, DEV>(P, first, wr, fin, fout, F, rho, uout, st);                         \
    }                                                                                                   \
    cudaError_t launch_stream_only_##SUF(const SimParams& P, const void* fin, void* fout,              \
                                         const void* rho, cudaStream_t st) {                           \
        return impl::stream_only<R, S>(P, fin, fout, rho, st);                                          \
    }                                                                                                   \
    cudaError_t launch_lbm_aa_##SUF(const SimParams& P, bool odd, bool wr, void* f, const void* F,     \
                                    void* rho, void* uout, cudaStream_t st) {                          \
        return impl::lbm_aa<R, S, DEV>(P, odd, wr, f, F, rho, uout, st);                                \
    }                                                                                                   \
    cudaError_t launch_aa_pop_out_##SUF(const SimParams& P, const void* f, const void* rho, double* dst, \
                                        int dir, cudaStream_t st) {                                    \
        return impl::aa_pop_out<R, S, DEV>(P, f, rho, dst, dir, st);                                    \
    }                                                                                                   \
    cudaError_t launch_swap_pairs_##SUF(const SimParams& P, void* f, cudaStream_t st) {                \
        return impl::swap_pairs<S>(P, f, st);                                                           \
    }                                                                                                   \
    cudaError_t launch_halo_merge_##SUF(const SimParams& P, void* f, const void* stage, int face,       \
                                        cudaStream_t st) {                                              \
        return impl::halo_merge<S>(P, f, stage, face, st);                                              \
    }                                                                                                   \
    cudaError_t launch_feq_init_##SUF(const SimParams& P, const void* rho, const void* u, void* f,     \
                                      cudaStream_t st) {                                               \
        return impl::feq_init<R, S, DEV>(P, rho, u, f, st);                                             \
    }                                                                                                   \
    cudaError_t launch_pop_in_##SUF(const SimParams& P, const double* src, void* dst, int dir,         \
                                    cudaStream_t st) {                                                 \
        return impl::pop_in<S, DEV>(P, src, dst, dir, st);                                              \
    }                                                                                                   \
    cudaError_t launch_pop_out_##SUF(const SimParams& P, const void* src, double* dst, int dir,        \
                                     cudaStream_t st) {                                                \
        return impl::pop_out<S, DEV>(P, src, dst, dir, st);                                             \
    }                                                                                                   \
    cudaError_t launch_real_in_##SUF(const double* src, void* dst, int64_t n, cudaStream_t st) {       \
        return impl::real_in<R>(src, dst, n, st);                                                       \
    }                                                                                                   \
    cudaError_t launch_real_out_##SUF(const void* src, double* dst, int64_t n, cudaStream_t st) {      \
        return impl::real_out<R>(src, dst, n, st);                                                      \
    }                                                                                                   \
    cudaError_t launch_flow_reduce_##SUF(const SimParams& P, const void* rho, const void* u,           \
                                         void* upast, double* partials, int G, cudaStream_t st) {      \
        return impl::flow_reduce<R>(P, rho, u, upast, partials, G, st);                                 \
    }                                                                                                   \
    cudaError_t launch_energy_reduce_##SUF(const SimParams& P, const void* q, double* partials, int G,  \
                                           cudaStream_t st) {                                          \
        return impl::energy_reduce<R>(P, q, partials, G, st);                                           \
    }                                                                                                   \
    cudaError_t launch_director_##SUF(const SimParams& P, const void* q, void* order, void* dir, int G, \
                                      cudaStream_t st) {                                               \
        return impl::director<R>(P, q, order, dir, G, st);                                              \
    }                                                                                                   \
    cudaError_t launch_defect_flags_##SUF(const SimParams& P, const void* dir, uint8_t* flags, int G,  \
                                          cudaStream_t st) {                                           \
        return impl::defect_flags<R>(P, dir, flags, G, st);                                             \
    }                                                                                                   \
    cudaError_t launch_defect_count_##SUF(const SimParams& P, const void* dir, double* partials, int G, \
                                          cudaStream_t st) {                                           \
        return impl::defect_count<R>(P, dir, partials, G, st);                                          \
    }                                                                                                   \
    cudaError_t launch_seeded_init_##SUF(const SimParams& P, uint64_t seed, double S0, double sigma,    \
                                         void* rho, void* u, void* q, void* F, cudaStream_t st) {      \
        return impl::seeded_init<R>(P, seed, S0, sigma, rho, u, q, F, st);                              \
    }                                                                                                   \
    cudaError_t launch_qsetup_##SUF(const SimParams& P, const void* qin, const void* uin, void* qout,   \
                                    void* sig, void* tau, void* F, cudaStream_t st) {                  \
        return impl::qsetup<R>(P, qin, uin, qout, sig, tau, F, st);                                     \
    }                                                                                                   \
    cudaError_t launch_active_force_##SUF(const SimParams& P, const void* q, const void* sig,           \
                                          const void* tau, const void* u, void* F, cudaStream_t st) {  \
        return impl::active_force<R>(P, q, sig, tau, u, F, st);                                         \
    }                                                                                                   \
    size_t qforce_smem_##SUF(const QTile& T) { return impl::qforce_smem<R>(T); }                       \
    int qforce_threads_##SUF(const QTile& T) { return impl::qforce_threads<R>(T); }                    \
    int march_blocks_##SUF(const SimParams& P, const LaunchShape& shape, bool fused_org) {             \
        return impl::march_blocks<R, S, DEV>(P, shape, fused_org);                                      \
    }                                                                                                   \
    cudaError_t prepare_##SUF(size_t max_smem) { return impl::prepare<R, S, DEV>(max_smem); }           \
    }
