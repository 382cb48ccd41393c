// qsplit.cuh -- the reference's Q stage as its two separate phases, for
// callers that replace the activity model between them (the virtual
// QTensorSolver::SetActiveStressAndComputeBodyForce, src/qtensor_solver.h:
// 11-21, 48).  The time step itself uses the one-pass z-marching kernel of
// qforce.cuh; these kernels serve the drop-in classes whose subclasses may
// override the second phase.
//
//   qsetup_kernel       StepAndSetupBodyForce (src/qtensor_solver.tpp:51-147):
//                       Q_new, Sigma, tau and the Ericksen seed of the body
//                       force, one thread per cell.
//   active_force_kernel the base SetActiveStressAndComputeBodyForce
//                       (src/qtensor_solver.tpp:155-217): grad Q_new with the
//                       wall ghosts, div(Sigma + tau) with the QXoff clamp,
//                       -ALPHA div Q_new and -MU u added to the force.
//
// Both use the point physics of physics.cuh in the reference's association
// order, so the FP64 instantiation (--fmad=false) is bitwise the reference.
#pragma once

#include "physics.cuh"

namespace lbman {

struct CellXYZ {
    int x, y, z;
    int64_t c;
};

__device__ __forceinline__ CellXYZ cell_xyz(const SimParams& P, int64_t c) {
    CellXYZ q;
    q.c = c;
    q.z = (int)(c / P.nxy);
    const int64_t r = c - (int64_t)q.z * P.nxy;
    q.y = (int)(r / P.nx);
    q.x = (int)(r - (int64_t)q.y * P.nx);
    return q;
}

// Offsets of the periodic-wrapped neighbours of a cell along each axis
// (a non-periodic wall's rule replaces the wrapped value where it applies).
struct NbrOff {
    int64_t xm, xp, ym, yp, zm, zp;
};

__device__ __forceinline__ NbrOff nbr_off(const SimParams& P, const CellXYZ& q) {
    NbrOff o;
    o.xm = q.x == 0 ? (int64_t)(P.nx - 1) : -1;
    o.xp = q.x == P.nx - 1 ? -(int64_t)(P.nx - 1) : 1;
    o.ym = q.y == 0 ? (int64_t)(P.ny - 1) * P.nx : -(int64_t)P.nx;
    o.yp = q.y == P.ny - 1 ? -(int64_t)(P.ny - 1) * P.nx : (int64_t)P.nx;
    o.zm = q.z == 0 ? (int64_t)(P.nz - 1) * P.nxy : -P.nxy;
    o.zp = q.z == P.nz - 1 ? -(int64_t)(P.nz - 1) * P.nxy : P.nxy;
    return o;
}

template <class R, bool UPWIND>
__global__ void __launch_bounds__(128) qsetup_kernel(const __grid_constant__ SimParams P, const R* __restrict__ qin,
                                                     const R* __restrict__ uin, R* __restrict__ qout,
                                                     R* __restrict__ sig, R* __restrict__ tau,
                                                     R* __restrict__ F) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.V) return;
    const int64_t V = P.V;
    const Phys<R>& K = phys_ref<R>(P);
    const CellXYZ q = cell_xyz(P, c);
    const NbrOff o = nbr_off(P, q);
    const AxisRule qx = q_rule(P, 0, q.x, P.nx), qy = q_rule(P, 1, q.y, P.ny), qz = q_rule(P, 2, q.z, P.nz);
    const VRule vx = v_rule(P, 0, q.x, P.nx), vy = v_rule(P, 1, q.y, P.ny), vz = v_rule(P, 2, q.z, P.nz);
    // QGradientAndLaplacian per component (src/boundary_handler.h:287-320)
    R Q[5];
    QD<R> d[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const R* a = qin + k * V + c;
        const R cc = a[0];
        R xm = a[o.xm], xp = a[o.xp], ym = a[o.ym], yp = a[o.yp], zm = a[o.zm], zp = a[o.zp];
        q_apply<R>(qx, K, k, cc, xm, xp);
        q_apply<R>(qy, K, k, cc, ym, yp);
        q_apply<R>(qz, K, k, cc, zm, zp);
        d[k] = q_derivs<R>(xm, xp, ym, yp, zm, zp, cc);
        Q[k] = cc;
    }
    // VelocityGradientTensor (src/boundary_handler.h:175-209): u_z,z is never formed
    const R u0[3] = {uin[c], uin[V + c], uin[2 * V + c]};
    R gr[8];
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) {
        const R* a = uin + comp * V + c;
        gr[comp * 3 + 0] = v_grad<R>(P, K, vx, comp, a[o.xm], u0[comp], a[o.xp], comp == 0);
        gr[comp * 3 + 1] = v_grad<R>(P, K, vy, comp, a[o.ym], u0[comp], a[o.yp], comp == 1);
        if (comp < 2) gr[comp * 3 + 2] = v_grad<R>(P, K, vz, comp, a[o.zm], u0[comp], a[o.zp], false);
    }
    GradU<R> g;
    g.ux_x = gr[0]; g.ux_y = gr[1]; g.ux_z = gr[2];
    g.uy_x = gr[3]; g.uy_y = gr[4]; g.uy_z = gr[5];
    g.uz_x = gr[6]; g.uz_y = gr[7];
    R qn[5], sg[5], ta[3], er[3];
    pointwise_q<R, UPWIND>(K, Q, u0[0], u0[1], u0[2], d, g, qn, sg, ta, er);
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        qout[k * V + c] = qn[k];
        sig[k * V + c] = sg[k];
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        tau[k * V + c] = ta[k];
        F[k * V + c] = er[k];
    }
}

template <class R>
__global__ void __launch_bounds__(128) active_force_kernel(const __grid_constant__ SimParams P, const R* __restrict__ q,
                                                           const R* __restrict__ sig, const R* __restrict__ tau,
                                                           const R* __restrict__ u, R* __restrict__ F) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.V) return;
    const int64_t V = P.V;
    const Phys<R>& K = phys_ref<R>(P);
    const CellXYZ p = cell_xyz(P, c);
    const NbrOff o = nbr_off(P, p);
    const AxisRule qx = q_rule(P, 0, p.x, P.nx), qy = q_rule(P, 1, p.y, P.ny), qz = q_rule(P, 2, p.z, P.nz);
    // grad Q with the wall ghosts (QGradientAndLaplacian on the current Q)
    R dQ[5][3];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const R* a = q + k * V + c;
        const R cc = a[0];
        R xm = a[o.xm], xp = a[o.xp], ym = a[o.ym], yp = a[o.yp], zm = a[o.zm], zp = a[o.zp];
        q_apply<R>(qx, K, k, cc, xm, xp);
        q_apply<R>(qy, K, k, cc, ym, yp);
        q_apply<R>(qz, K, k, cc, zm, zp);
        dQ[k][0] = R(0.5) * (xp - xm);
        dQ[k][1] = R(0.5) * (yp - ym);
        dQ[k][2] = R(0.5) * (zp - zm);
    }
    // PassiveStressDivergence (src/boundary_handler.h:335-392): differences
    // with the Neumann/periodic index clamp QXoff (src/offsets.h:59-83)
    const bool xmc = p.x == 0 && !P.qper[0], xpc = p.x == P.nx - 1 && !P.qper[1];
    const bool ymc = p.y == 0 && !P.qper[2], ypc = p.y == P.ny - 1 && !P.qper[3];
    const bool zmc = p.z == 0 && !P.qper[4], zpc = p.z == P.nz - 1 && !P.qper[5];
    R dS[3][5], dT[3][3];
#pragma unroll
    for (int v = 0; v < 8; ++v) {
        const R* a = (v < 5 ? sig + v * V : tau + (v - 5) * V) + c;
        const R cc = a[0];
        const R xm = xmc ? cc : a[o.xm], xp = xpc ? cc : a[o.xp];
        const R ym = ymc ? cc : a[o.ym], yp = ypc ? cc : a[o.yp];
        const R zm = zmc ? cc : a[o.zm], zp = zpc ? cc : a[o.zp];
        const R ddx = R(0.5) * (xp - xm), ddy = R(0.5) * (yp - ym), ddz = R(0.5) * (zp - zm);
        if (v < 5) { dS[0][v] = ddx; dS[1][v] = ddy; dS[2][v] = ddz; }
        else { dT[0][v - 5] = ddx; dT[1][v - 5] = ddy; dT[2][v - 5] = ddz; }
    }
    // F += force (the reference adds to the Ericksen seed already in F)
    const R seed[3] = {F[c], F[V + c], F[2 * V + c]};
    R out[3];
    active_passive_force<R>(K, dQ, dS, dT, u[c], u[V + c], u[2 * V + c], seed, out);
#pragma unroll
    for (int k = 0; k < 3; ++k) F[k * V + c] = out[k];
}

}  // namespace lbman
