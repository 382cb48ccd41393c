// ens.cuh -- ensemble kernels: many independent boxes of different sizes,
// boundary configurations and physical parameters advanced together.
//
// Every box is described by an EnsBox in device memory (its own SimParams
// and field pointers).  The host flattens all boxes into work lists -- one
// item per z-marching block of the Q+force kernel, one per 256-cell block of
// the LBM kernel -- and each launch covers every box: a persistent grid of
// blocks strides through the list, running the same march / gather-collide
// code as the single-box kernels on the item's box.  A time step of the whole
// ensemble is therefore one launch per kernel (two in the split organisation,
// one fused), which the host replays from a CUDA graph.  There is no
// communication between boxes.
#pragma once

#include "fused.cuh"
#include "lbm.cuh"

namespace lbman {

struct EnsBox {
    SimParams P;
    FastDiv dnx, dnxy;
    void* q[2];   // Q, double buffered
    void* u[2];   // u, double buffered (fused); the split organisation uses u[0] only
    void* f[2];   // populations, double buffered
    void* rho;
    void* F;
    int zc;       // z chunk of this box's Q work items
};

struct EnsQWork {
    int box, bx, by, bz;
};
struct EnsLbmWork {
    int box, block;
};

template <class TL, class R, bool UPWIND>
__global__ void __launch_bounds__(TL::NT, (Stage<TL, R>::MINB)) ens_qforce_kernel(const EnsBox* __restrict__ boxes,
                                                            const EnsQWork* __restrict__ work, int nwork,
                                                            int par) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    // The item's box parameters, copied to shared memory once per item: the
    // z march reads them throughout, and a global-memory copy would cost a
    // load per use where a single-box launch reads its constant bank.  Every
    // tile whose staging fits one block (227 KB) leaves room for the copy
    // (largest: FP64 32x8, 216 672 B staging + 1 368 B of parameters).
    static_assert(Stage<TL, R>::bytes + sizeof(SimParams) + 1024 <= 227 * 1024,
                  "the box parameters must fit beside the tile's staging");
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const EnsQWork it = work[w];
        const EnsBox& B = boxes[it.box];
        const int z0 = it.bz * B.zc;
        __shared__ __align__(16) uint32_t pbuf[sizeof(SimParams) / 4];
        const SimParams& Ps = *reinterpret_cast<const SimParams*>(pbuf);
        const uint32_t* src = reinterpret_cast<const uint32_t*>(&B.P);
        for (int i = threadIdx.x; i < (int)(sizeof(SimParams) / 4); i += blockDim.x) pbuf[i] = src[i];
        __syncthreads();
        if (z0 < Ps.nz)
            qf_march<TL, R, UPWIND>(Ps, it.bx * TL::TCX, it.by * TL::TCY, z0, min(z0 + B.zc, Ps.nz),
                                    (const R*)B.q[par], (const R*)B.u[0], reinterpret_cast<R*>(smem_raw),
                                    StoreQForce<R>{(R*)B.q[1 - par], (R*)B.F, Ps.V});
        __syncthreads();  // the staging rings and the parameters are reused by the next item
    }
}

template <class TL, class R, class S, bool DEV, bool UPWIND>
__global__ void __launch_bounds__(TL::NT) ens_fused_kernel(const EnsBox* __restrict__ boxes,
                                                           const EnsQWork* __restrict__ work, int nwork, int par,
                                                           int first, int write_rho_all) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const EnsQWork it = work[w];
        const EnsBox& B = boxes[it.box];
        const int z0 = it.bz * B.zc;
        if (z0 < B.P.nz)
            qf_march<TL, R, UPWIND>(B.P, it.bx * TL::TCX, it.by * TL::TCY, z0, min(z0 + B.zc, B.P.nz),
                                    (const R*)B.q[par], (const R*)B.u[par], reinterpret_cast<R*>(smem_raw),
                                    CollideCell<R, S, DEV>{B.P, phys_ref<R>(B.P), first, (R*)B.q[1 - par],
                                                           (R*)B.u[1 - par], (const S*)B.f[par],
                                                           (S*)B.f[1 - par], (R*)B.rho, nullptr, write_rho_all});
        __syncthreads();
    }
}

// Held to the single-box walled LBM kernel's register budget (5 blocks per SM
// for FP32 compute, 2 for FP64); each work item's box picks the periodic or the
// walled gather (block-uniform).
template <class R, class S, bool DEV>
__global__ void __launch_bounds__(256, lbm_min_blocks<R, S, true>()) ens_lbm_kernel(const EnsBox* __restrict__ boxes,
                                                      const EnsLbmWork* __restrict__ work, int nwork, int par,
                                                      int first, int write_rho_all) {
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        const EnsLbmWork it = work[w];
        const EnsBox& B = boxes[it.box];
        const SimParams& P = B.P;
        const int64_t c = (int64_t)it.block * blockDim.x + threadIdx.x;
        if (c >= P.V) continue;
        const int64_t V = P.V;
        const Phys<R>& K = phys_ref<R>(P);
        CellPos q;
        q.z = (int)fdiv((uint32_t)c, B.dnxy);
        const uint32_t r = (uint32_t)(c - (int64_t)q.z * P.nxy);
        q.y = (int)fdiv(r, B.dnx);
        q.x = (int)(r - (uint32_t)q.y * (uint32_t)P.nx);
        const bool mv = P.moving_any && touches_moving(P, q.x, q.y, q.z);
        R* rho_buf = (R*)B.rho;
        const R* F = (const R*)B.F;
        R f[15];
        if (P.uper[0] && P.uper[2] && P.uper[4])
            load_pre<R, S, false>(P, K, first != 0, (const S*)B.f[par], c, q, R(0), f);
        else
            load_pre<R, S, true>(P, K, first != 0, (const S*)B.f[par], c, q, (mv && !first) ? rho_buf[c] : R(0), f);
        R rho, ux, uy, uz;
        collide<R, DEV>(K, f, F[c], F[V + c], F[2 * V + c], rho, ux, uy, uz);
        S* fout = (S*)B.f[1 - par];
#pragma unroll
        for (int j = 0; j < 15; ++j) Store<S>::st(fout + j * V + c, f[j]);
        R* u = (R*)B.u[0];
        u[c] = ux;
        u[V + c] = uy;
        u[2 * V + c] = uz;
        if (write_rho_all || mv) rho_buf[c] = rho;
    }
}

}  // namespace lbman
