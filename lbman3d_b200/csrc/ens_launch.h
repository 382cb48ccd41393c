// ens_launch.h -- host-side launchers of the ensemble kernels (kernels_ens.cu).
#pragma once

#include <cuda_runtime.h>

#include "ens.cuh"

namespace lbman {

// One Q+force (or fused) launch over every box of an ensemble.
struct EnsQLaunch {
    const EnsBox* boxes;
    const EnsQWork* work;
    int nwork;
    int tcx, tcy;
    bool fused, upwind;
    int par, first, write_rho_all;
    int grid;
};

#define LBMAN_ENS_DECLARE(SUF)                                                                           \
    cudaError_t ens_qstep_##SUF(const EnsQLaunch& L, cudaStream_t st);                                   \
    cudaError_t ens_lbm_##SUF(const EnsBox* b, const EnsLbmWork* w, int n, int par, int first, int wr, int grid, \
                              cudaStream_t st);                                                          \
    cudaError_t ens_prepare_##SUF(size_t max_smem);                                                      \
    int ens_blocks_per_sm_##SUF(int tcx, int tcy, bool fused);

LBMAN_ENS_DECLARE(f64)
LBMAN_ENS_DECLARE(f32)
LBMAN_ENS_DECLARE(f16)

}  // namespace lbman
