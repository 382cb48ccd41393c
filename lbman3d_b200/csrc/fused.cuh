// fused.cuh -- a whole time step in one kernel: the Q-tensor update with the
// full body force (qforce.cuh) immediately followed, cell by cell, by the
// D3Q15 gather/collide (lbm.cuh), with the body force kept in registers.
//
// This is the merge the reference's own design note asks for
// (src/qtensor_solver.tpp:219-248) carried one step further: per cell the
// step reads f* (15), Q (5) and u (3) and writes f* (15), Q_new (5) and
// u (3) -- 46 words, the compulsory state traffic -- while the reference's
// three kernels move 83.  Q and u are double buffered (blocks read their
// neighbours' old values while writing new ones); rho is written only where
// a moving wall needs it next step, or everywhere on request, and the body
// force only on request (Fout != nullptr).
#pragma once

#include "lbm.cuh"
#include "qforce.cuh"

namespace lbman {

// Consumer of the fused organisation: store Q_new (and F on request), then
// gather, collide and store this cell's populations, velocity and density.
template <class R, class S, bool DEV>
struct CollideCell {
    const SimParams& P;
    const Phys<R>& K;
    int first;
    R* __restrict__ qout;
    R* __restrict__ uout;
    const S* __restrict__ fin;
    S* __restrict__ fout;
    R* __restrict__ rho_buf;
    R* __restrict__ Fout;
    int write_rho_all;
    __device__ __forceinline__ void operator()(int64_t cell, int x, int y, int z, const R qn[5], const R F[3],
                                               const R*) const {
        const int64_t V = P.V;
#pragma unroll
        for (int k = 0; k < 5; ++k) qout[k * V + cell] = qn[k];
        if (Fout) {
            Fout[cell] = F[0];
            Fout[V + cell] = F[1];
            Fout[2 * V + cell] = F[2];
        }
        const bool mv = P.moving_any && touches_moving(P, x, y, z);
        R f[15];
        load_pre<R, S>(P, K, first != 0, fin, cell, CellPos{x, y, z}, (mv && !first) ? rho_buf[cell] : R(0), f);
        R rho, ux, uy, uz;
        collide<R, DEV>(K, f, F[0], F[1], F[2], rho, ux, uy, uz);
#pragma unroll
        for (int j = 0; j < 15; ++j) Store<S>::st(fout + j * V + cell, f[j]);
        uout[cell] = ux;
        uout[V + cell] = uy;
        uout[2 * V + cell] = uz;
        if (write_rho_all || mv) rho_buf[cell] = rho;
    }
};

template <class TL, class R, class S, bool DEV, bool UPWIND>
__global__ void __launch_bounds__(TL::NT) fused_kernel(const __grid_constant__ SimParams P, int zc_len, int first,
                                                       const R* __restrict__ qin, const R* __restrict__ uin,
                                                       R* __restrict__ qout, R* __restrict__ uout,
                                                       const S* __restrict__ fin, S* __restrict__ fout,
                                                       R* __restrict__ rho_buf, R* __restrict__ Fout,
                                                       int write_rho_all) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    qf_run<TL, R, UPWIND>(
        P, zc_len, qin, uin, reinterpret_cast<R*>(smem_raw),
        CollideCell<R, S, DEV>{P, phys_ref<R>(P), first, qout, uout, fin, fout, rho_buf, Fout, write_rho_all});
}

}  // namespace lbman
