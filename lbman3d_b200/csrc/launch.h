// launch.h -- host-side launchers of the sm_100a kernels, one set per
// precision.  kernels_f64.cu (compiled with --fmad=false so the FP64 path
// reproduces the reference's arithmetic bit for bit) defines the *_f64
// functions; kernels_f32.cu defines *_f32 (FP32 storage) and *_f16 (FP16
// population storage, FP32 compute).
#pragma once

#include <cuda_runtime.h>

#include "common.cuh"

namespace lbman {

// Work shape of one step; filled by the host layer from the grid size and the
// autotuner.
struct LaunchShape {
    QTile tile;        // tile.zc == 0: balanced one-wave schedule
    int qthreads;
    int num_sms = 148;  // multiprocessors of the device (sizes the balanced grid)
};

#define LBMAN_DECLARE_LAUNCHERS(SUF)                                                                   \
    cudaError_t launch_qforce_##SUF(const SimParams& P, const LaunchShape& S, const void* qin,          \
                                    const void* uin, void* qout, void* Fout, cudaStream_t st);         \
    cudaError_t launch_fused_##SUF(const SimParams& P, const LaunchShape& S, bool first,                \
                                   const void* qin, const void* uin, void* qout, void* uout,           \
                                   const void* fin, void* fout, void* rho, void* Fout,                 \
                                   bool write_rho_all, cudaStream_t st);                               \
    cudaError_t launch_lbm_##SUF(const SimParams& P, bool first, bool write_rho_all, const void* fin,  \
                                 void* fout, const void* F, void* rho, void* uout, cudaStream_t st);   \
    cudaError_t launch_stream_only_##SUF(const SimParams& P, const void* fin, void* fout,              \
                                         const void* rho, cudaStream_t st);                            \
    cudaError_t launch_lbm_aa_##SUF(const SimParams& P, bool odd, bool write_rho_all, void* f,         \
                                    const void* F, void* rho, void* uout, cudaStream_t st);            \
    cudaError_t launch_aa_pop_out_##SUF(const SimParams& P, const void* f, const void* rho, double* dst, \
                                        int dir, cudaStream_t st);                                     \
    cudaError_t launch_swap_pairs_##SUF(const SimParams& P, void* f, cudaStream_t st);                 \
    cudaError_t launch_halo_merge_##SUF(const SimParams& P, void* f, const void* stage, int face,      \
                                        cudaStream_t st);                                              \
    cudaError_t launch_feq_init_##SUF(const SimParams& P, const void* rho, const void* u, void* f,     \
                                      cudaStream_t st);                                                \
    cudaError_t launch_pop_in_##SUF(const SimParams& P, const double* src, void* dst, int dir,         \
                                    cudaStream_t st);                                                  \
    cudaError_t launch_pop_out_##SUF(const SimParams& P, const void* src, double* dst, int dir,        \
                                     cudaStream_t st);                                                 \
    cudaError_t launch_real_in_##SUF(const double* src, void* dst, int64_t n, cudaStream_t st);        \
    cudaError_t launch_real_out_##SUF(const void* src, double* dst, int64_t n, cudaStream_t st);       \
    cudaError_t launch_flow_reduce_##SUF(const SimParams& P, const void* rho, const void* u,           \
                                         void* upast, double* partials, int G, cudaStream_t st);       \
    cudaError_t launch_energy_reduce_##SUF(const SimParams& P, const void* q, double* partials, int G,  \
                                           cudaStream_t st);                                           \
    cudaError_t launch_director_##SUF(const SimParams& P, const void* q, void* order, void* dir, int G, \
                                      cudaStream_t st);                                                \
    cudaError_t launch_defect_flags_##SUF(const SimParams& P, const void* dir, uint8_t* flags, int G,  \
                                          cudaStream_t st);                                            \
    cudaError_t launch_defect_count_##SUF(const SimParams& P, const void* dir, double* partials, int G, \
                                          cudaStream_t st);                                            \
    cudaError_t launch_seeded_init_##SUF(const SimParams& P, uint64_t seed, double S0, double sigma,    \
                                         void* rho, void* u, void* q, void* F, cudaStream_t st);       \
    cudaError_t launch_qsetup_##SUF(const SimParams& P, const void* qin, const void* uin, void* qout,   \
                                    void* sig, void* tau, void* F, cudaStream_t st);                   \
    cudaError_t launch_active_force_##SUF(const SimParams& P, const void* q, const void* sig,           \
                                          const void* tau, const void* u, void* F, cudaStream_t st);   \
    size_t qforce_smem_##SUF(const QTile& T);                                                          \
    int qforce_threads_##SUF(const QTile& T);                                                          \
    int march_blocks_##SUF(const SimParams& P, const LaunchShape& shape, bool fused_org);              \
    cudaError_t prepare_##SUF(size_t max_smem);

LBMAN_DECLARE_LAUNCHERS(f64)
LBMAN_DECLARE_LAUNCHERS(f32)
LBMAN_DECLARE_LAUNCHERS(f16)

cudaError_t launch_fold(const double* partials, int G, int nq, int nmax, double* out, cudaStream_t st);

}  // namespace lbman
