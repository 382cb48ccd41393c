// ens_impl.cuh -- launchers of the ensemble kernels (ens.cuh), instantiated
// by kernels_ens.cu (FP32, FP16 storage) and kernels_ens_f64.cu (FP64, built
// with --fmad=false like the single-box FP64 path, so batched and single-box
// FP64 runs agree bit for bit).  Grids are persistent: as many blocks as fit
// on the device at once, striding through the work lists.
#pragma once
#include "ens.cuh"
#include "ens_launch.h"
#include "kernels_impl.cuh"

namespace lbman {
namespace {

template <class R, class S, bool DEV>
struct EnsImpl {
    // Resident blocks per SM of the persistent Q (or fused) grid: the larger
    // of the occupancy query and the count from the SM's resources (the query
    // has answered low for kernels that run two blocks per SM here).
    template <class TL>
    static int occupancy(bool fused) {
        int n = 0;
        const size_t smem = TL::template smem_bytes<R>();
        if (fused) {
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ens_fused_kernel<TL, R, S, DEV, false>, TL::NT,
                                                              smem) != cudaSuccess)
                cudaGetLastError();
            n = std::max(n, impl::fit_blocks<ens_fused_kernel<TL, R, S, DEV, false>>(TL::NT, smem));
        } else {
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, ens_qforce_kernel<TL, R, false>, TL::NT, smem) !=
                cudaSuccess)
                cudaGetLastError();
            n = std::max(n, impl::fit_blocks<ens_qforce_kernel<TL, R, false>>(TL::NT, smem));
        }
        return n;
    }

    static cudaError_t qstep(const EnsQLaunch& L, cudaStream_t st) {
        return impl::with_tile<R>(L.tcx, L.tcy, [&](auto tl) {
            using TL = decltype(tl);
            const size_t smem = TL::template smem_bytes<R>();
            if (L.fused) {
                auto go = [&](auto kern) {
                    kern<<<L.grid, TL::NT, smem, st>>>(L.boxes, L.work, L.nwork, L.par, L.first, L.write_rho_all);
                };
                if (L.upwind) go(ens_fused_kernel<TL, R, S, DEV, true>);
                else go(ens_fused_kernel<TL, R, S, DEV, false>);
            } else {
                if (L.upwind)
                    ens_qforce_kernel<TL, R, true><<<L.grid, TL::NT, smem, st>>>(L.boxes, L.work, L.nwork, L.par);
                else
                    ens_qforce_kernel<TL, R, false><<<L.grid, TL::NT, smem, st>>>(L.boxes, L.work, L.nwork, L.par);
            }
            return cudaGetLastError();
        });
    }

    static cudaError_t lbm(const EnsBox* boxes, const EnsLbmWork* work, int nwork, int par, int first, int wr,
                           int grid, cudaStream_t st) {
        ens_lbm_kernel<R, S, DEV><<<grid, 256, 0, st>>>(boxes, work, nwork, par, first, wr);
        return cudaGetLastError();
    }

    static cudaError_t prepare(size_t max_smem) {
        cudaError_t e = cudaSuccess;
        for (const auto& xy : kTileList) {
            const int x = xy[0], y = xy[1];
            impl::with_tile<R>(x, y, [&](auto tl) {
                using TL = decltype(tl);
                // the tile's own staging (the Q kernel may also hold static
                // shared memory, so the device maximum would not fit)
                const size_t need = std::min(max_smem, TL::template smem_bytes<R>());
                auto attr = [&](auto kern) {
                    if (e == cudaSuccess)
                        e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)need);
                };
                attr(ens_qforce_kernel<TL, R, true>);
                attr(ens_qforce_kernel<TL, R, false>);
                attr(ens_fused_kernel<TL, R, S, DEV, true>);
                attr(ens_fused_kernel<TL, R, S, DEV, false>);
                return cudaSuccess;
            });
        }
        return e;
    }

    static int blocks_per_sm(int tcx, int tcy, bool fused) {
        int n = 0;
        impl::with_tile<R>(tcx, tcy, [&](auto tl) {
            n = occupancy<decltype(tl)>(fused);
            return cudaSuccess;
        });
        return n;
    }
};

}  // namespace

}  // namespace lbman

#define LBMAN_ENS_DEFINE(SUF, R, S, DEV)                                                                 \
    namespace lbman {                                                                                     \
    LBMAN_ENS_DEFINE_BODY(SUF, R, S, DEV)                                                                 \
    }

namespace lbman {
#define LBMAN_ENS_DEFINE_BODY(SUF, R, S, DEV)                                                                 \
    cudaError_t ens_qstep_##SUF(const EnsQLaunch& L, cudaStream_t st) { return EnsImpl<R, S, DEV>::qstep(L, st); } \
    cudaError_t ens_lbm_##SUF(const EnsBox* b, const EnsLbmWork* w, int n, int par, int first, int wr, int grid, \
                              cudaStream_t st) {                                                          \
        return EnsImpl<R, S, DEV>::lbm(b, w, n, par, first, wr, grid, st);                                \
    }                                                                                                     \
    cudaError_t ens_prepare_##SUF(size_t s) { return EnsImpl<R, S, DEV>::prepare(s); }                    \
    int ens_blocks_per_sm_##SUF(int x, int y, bool fused) { return EnsImpl<R, S, DEV>::blocks_per_sm(x, y, fused); }

}  // namespace lbman
