// qforce.cuh -- one kernel for the whole Q-tensor half of a time step:
// QTensorSolver::StepAndSetupBodyForce followed by
// SetActiveStressAndComputeBodyForce (src/qtensor_solver.tpp:51-217), i.e.
// the reference's GpuQTensorStep + GpuComputeBodyForce pair
// (src/cuda/kernels.cu:122-292) in a single pass.
//
// Each block owns a tcx x tcy tile of the x-y plane and marches through a
// chunk of z planes.  Q and u (8 values per cell) are staged in shared
// memory as a ring of three planes with a 2-cell x-y halo; the per-cell
// results Q_new, Sigma, tau and the Ericksen force (16 values) are kept as a
// ring of three planes with a 1-cell halo.  The stress divergence and the
// gradient of Q_new are then taken from shared memory, so Sigma, tau, Q_new
// and the Ericksen seed never travel through HBM: per cell the kernel reads
// Q, u once and writes Q_new and the body force F once (16 words), instead
// of the reference's 46 words across two kernels.
//
// Halo cells are loaded with periodic wrap on every axis; the wall rules
// then choose between the wrapped image, the centre value (clamp) and the
// anchoring ghost exactly as the reference's index/ghost policies do, so a
// wrapped value is only ever used on a periodic side.
#pragma once

#include "physics.cuh"

namespace lbman {

// Ring slots: results (B) keep 3 planes, staged Q/u keep 4 (one is in flight).
__device__ __forceinline__ int ring3(int z, int z0) { return (z - z0 + 6) % 3; }
__device__ __forceinline__ int ring4(int z, int z0) { return (z - z0 + 8) & 3; }

// Asynchronous global->shared copies (cp.async, completion via wait_all).
__device__ __forceinline__ void cp_async(float* s, const float* g) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((unsigned)__cvta_generic_to_shared(s)),
                 "l"(g));
}
__device__ __forceinline__ void cp_async(double* s, const double* g) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((unsigned)__cvta_generic_to_shared(s)),
                 "l"(g));
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Issue the copies of plane zg (Q then u, tile + 2-cell halo, periodic wrap)
// into its ring slot.  Completes at the next cp_async_wait_all().
template <class R>
__device__ __forceinline__ void qf_load_plane(const SimParams& P, const QTile& T, int x0, int y0,
                                              int z0, int zg, const R* __restrict__ qin,
                                              const R* __restrict__ uin, R* QU) {
    const int uxw = T.tcx + 4, uyw = T.tcy + 4, nQU = uxw * uyw;
    const int zw = wrap_coord(zg, P.nz);
    R* dst = QU + ring4(zg, z0) * 8 * nQU;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
    const int64_t zoff = (int64_t)zw * P.nxy;
    for (int row = warp; row < 8 * uyw; row += nwarp) {
        const int var = row / uyw, ly = row - var * uyw;
        const int gy = wrap_coord(y0 - 2 + ly, P.ny);
        const R* src = (var < 5 ? qin + (int64_t)var * P.V : uin + (int64_t)(var - 5) * P.V) + zoff +
                       (int64_t)gy * P.nx;
        R* d = dst + var * nQU + ly * uxw;
        for (int lx = lane; lx < uxw; lx += 32) cp_async(d + lx, src + wrap_coord(x0 - 2 + lx, P.nx));
    }
}

template <class R, bool UPWIND>
__device__ __forceinline__ void qf_compute_plane(const SimParams& P, const QTile& T, int x0, int y0,
                                                 int z0, int zb, const R* QU, R* Bs) {
    const int uxw = T.tcx + 4, uyw = T.tcy + 4, nQU = uxw * uyw;
    const int bxw = T.tcx + 2, byw = T.tcy + 2, nB = bxw * byw;
    const R* Qc = QU + ring4(zb, z0) * 8 * nQU;
    const R* Qm = QU + ring4(zb - 1, z0) * 8 * nQU;
    const R* Qp = QU + ring4(zb + 1, z0) * 8 * nQU;
    R* Bd = Bs + ring3(zb, z0) * 16 * nB;
    const int az = wrap_coord(zb, P.nz);
    for (int p = threadIdx.x; p < nB; p += blockDim.x) {
        const int lby = p / bxw, lbx = p - lby * bxw;
        const int ax = wrap_coord(x0 - 1 + lbx, P.nx), ay = wrap_coord(y0 - 1 + lby, P.ny);
        const int up = (lby + 1) * uxw + lbx + 1;
        R Q[5];
        QD<R> d[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            const R* qc = Qc + k * nQU;
            const R c = qc[up];
            R xm, xp, ym, yp, zm, zp;
            q_pair<R>(P, 0, k, ax, P.nx, qc[up - 1], c, qc[up + 1], xm, xp);
            q_pair<R>(P, 1, k, ay, P.ny, qc[up - uxw], c, qc[up + uxw], ym, yp);
            q_pair<R>(P, 2, k, az, P.nz, Qm[k * nQU + up], c, Qp[k * nQU + up], zm, zp);
            d[k] = q_derivs<R>(xm, xp, ym, yp, zm, zp, c);
            Q[k] = c;
        }
        const R* uxc = Qc + 5 * nQU;
        const R* uyc = Qc + 6 * nQU;
        const R* uzc = Qc + 7 * nQU;
        const R ux0 = uxc[up], uy0 = uyc[up], uz0 = uzc[up];
        GradU<R> g;
        g.ux_x = v_grad<R>(P, 0, 0, ax, P.nx, uxc[up - 1], ux0, uxc[up + 1], true);
        g.ux_y = v_grad<R>(P, 1, 0, ay, P.ny, uxc[up - uxw], ux0, uxc[up + uxw], false);
        g.ux_z = v_grad<R>(P, 2, 0, az, P.nz, Qm[5 * nQU + up], ux0, Qp[5 * nQU + up], false);
        g.uy_x = v_grad<R>(P, 0, 1, ax, P.nx, uyc[up - 1], uy0, uyc[up + 1], false);
        g.uy_y = v_grad<R>(P, 1, 1, ay, P.ny, uyc[up - uxw], uy0, uyc[up + uxw], true);
        g.uy_z = v_grad<R>(P, 2, 1, az, P.nz, Qm[6 * nQU + up], uy0, Qp[6 * nQU + up], false);
        g.uz_x = v_grad<R>(P, 0, 2, ax, P.nx, uzc[up - 1], uz0, uzc[up + 1], false);
        g.uz_y = v_grad<R>(P, 1, 2, ay, P.ny, uzc[up - uxw], uz0, uzc[up + uxw], false);
        R qn[5], sg[5], ta[3], er[3];
        pointwise_q<R, UPWIND>(P, Q, ux0, uy0, uz0, d, g, qn, sg, ta, er);
#pragma unroll
        for (int k = 0; k < 5; ++k) Bd[k * nB + p] = qn[k];
#pragma unroll
        for (int k = 0; k < 5; ++k) Bd[(5 + k) * nB + p] = sg[k];
#pragma unroll
        for (int k = 0; k < 3; ++k) Bd[(10 + k) * nB + p] = ta[k];
#pragma unroll
        for (int k = 0; k < 3; ++k) Bd[(13 + k) * nB + p] = er[k];
    }
}

// Body force at the tile cells of plane zc, from the staged B planes.
// OutFn(cell, x, y, z, qn[5], F[3], u[3]) consumes the result (stores it, or
// runs the collide/stream step on it in the fused kernel).
template <class R, class OutFn>
__device__ __forceinline__ void qf_force_plane(const SimParams& P, const QTile& T, int x0, int y0,
                                               int z0, int zc, const R* QU, const R* Bs, OutFn&& out) {
    const int uxw = T.tcx + 4, uyw = T.tcy + 4, nQU = uxw * uyw;
    const int bxw = T.tcx + 2, byw = T.tcy + 2, nB = bxw * byw;
    const R* B0 = Bs + ring3(zc, z0) * 16 * nB;
    const R* Bm = Bs + ring3(zc - 1, z0) * 16 * nB;
    const R* Bp = Bs + ring3(zc + 1, z0) * 16 * nB;
    const R* U0 = QU + ring4(zc, z0) * 8 * nQU;
    const int ntile = T.tcx * T.tcy;
    for (int p = threadIdx.x; p < ntile; p += blockDim.x) {
        const int lcy = p / T.tcx, lcx = p - lcy * T.tcx;
        const int gx = x0 + lcx, gy = y0 + lcy;
        if (gx >= P.nx || gy >= P.ny) continue;
        const int bp = (lcy + 1) * bxw + lcx + 1;
        // grad Q_new with the wall ghosts (QGradientAndLaplacian on the new Q).
        R dQ[5][3];
        R qn[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            const R* b = B0 + k * nB;
            const R c = b[bp];
            qn[k] = c;
            R m, q;
            q_pair<R>(P, 0, k, gx, P.nx, b[bp - 1], c, b[bp + 1], m, q);
            dQ[k][0] = (q - m) / R(2.0);
            q_pair<R>(P, 1, k, gy, P.ny, b[bp - bxw], c, b[bp + bxw], m, q);
            dQ[k][1] = (q - m) / R(2.0);
            q_pair<R>(P, 2, k, zc, P.nz, Bm[k * nB + bp], c, Bp[k * nB + bp], m, q);
            dQ[k][2] = (q - m) / R(2.0);
        }
        // Sigma / tau differences with the Neumann/periodic index clamp QXoff
        // (src/offsets.h:59-83, used by PassiveStressDivergence).
        const bool xmc = gx == 0 && !P.qper[0], xpc = gx == P.nx - 1 && !P.qper[1];
        const bool ymc = gy == 0 && !P.qper[2], ypc = gy == P.ny - 1 && !P.qper[3];
        const bool zmc = zc == 0 && !P.qper[4], zpc = zc == P.nz - 1 && !P.qper[5];
        R dS[3][5], dT[3][3];
#pragma unroll
        for (int v = 0; v < 8; ++v) {
            const R* b = B0 + (5 + v) * nB;
            const R c = b[bp];
            const R xm = xmc ? c : b[bp - 1], xp = xpc ? c : b[bp + 1];
            const R ym = ymc ? c : b[bp - bxw], yp = ypc ? c : b[bp + bxw];
            const R zm = zmc ? c : Bm[(5 + v) * nB + bp], zp = zpc ? c : Bp[(5 + v) * nB + bp];
            const R ddx = (xp - xm) / R(2.0), ddy = (yp - ym) / R(2.0), ddz = (zp - zm) / R(2.0);
            if (v < 5) { dS[0][v] = ddx; dS[1][v] = ddy; dS[2][v] = ddz; }
            else { dT[0][v - 5] = ddx; dT[1][v - 5] = ddy; dT[2][v - 5] = ddz; }
        }
        const int uq = (lcy + 2) * uxw + lcx + 2;
        const R u[3] = {U0[5 * nQU + uq], U0[6 * nQU + uq], U0[7 * nQU + uq]};
        const R er[3] = {B0[13 * nB + bp], B0[14 * nB + bp], B0[15 * nB + bp]};
        R F[3];
        active_passive_force<R>(P, dQ, dS, dT, u[0], u[1], u[2], er, F);
        const int64_t cell = (int64_t)zc * P.nxy + (int64_t)gy * P.nx + gx;
        out(cell, gx, gy, zc, qn, F, u);
    }
}

// Marches a block through its z chunk; PlaneOut is called once per output
// plane after the staged planes are complete.  The copy of plane zc+3 is in
// flight while planes zc+1 (results) and zc (force, output) are computed, so
// the global-memory latency of the staging is hidden behind the arithmetic.
template <class R, bool UPWIND, class PlaneOut>
__device__ __forceinline__ void qf_march(const SimParams& P, const QTile& T,
                                         const R* __restrict__ qin, const R* __restrict__ uin,
                                         R* QU, R* Bs, PlaneOut&& plane_out) {
    const int x0 = blockIdx.x * T.tcx, y0 = blockIdx.y * T.tcy;
    const int z0 = blockIdx.z * T.zc;
    if (z0 >= P.nz) return;
    const int z1 = min(z0 + T.zc, P.nz);
    for (int z = z0 - 2; z <= z0 + 1; ++z) qf_load_plane<R>(P, T, x0, y0, z0, z, qin, uin, QU);
    cp_async_wait_all();
    __syncthreads();
    qf_compute_plane<R, UPWIND>(P, T, x0, y0, z0, z0 - 1, QU, Bs);
    qf_compute_plane<R, UPWIND>(P, T, x0, y0, z0, z0, QU, Bs);
    __syncthreads();  // slot of z0-2 is free again
    qf_load_plane<R>(P, T, x0, y0, z0, z0 + 2, qin, uin, QU);
    cp_async_wait_all();
    __syncthreads();
    for (int zc = z0; zc < z1; ++zc) {
        // slot of zc-1 was last read by the previous iteration (before its final barrier)
        if (zc + 1 < z1) qf_load_plane<R>(P, T, x0, y0, z0, zc + 3, qin, uin, QU);
        qf_compute_plane<R, UPWIND>(P, T, x0, y0, z0, zc + 1, QU, Bs);
        __syncthreads();
        plane_out(x0, y0, z0, zc);
        cp_async_wait_all();
        __syncthreads();
    }
}

template <class R>
__host__ __device__ inline int qf_qu_elems(const QTile& T) {
    return 4 * 8 * (T.tcx + 4) * (T.tcy + 4);
}

template <class R, bool UPWIND>
__global__ void __launch_bounds__(512) qforce_kernel(SimParams P, QTile T, const R* __restrict__ qin,
                                                     const R* __restrict__ uin, R* __restrict__ qout,
                                                     R* __restrict__ Fout) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R* QU = reinterpret_cast<R*>(smem_raw);
    R* Bs = QU + qf_qu_elems<R>(T);
    const int64_t V = P.V;
    qf_march<R, UPWIND>(P, T, qin, uin, QU, Bs, [&](int x0, int y0, int z0, int zc) {
        qf_force_plane<R>(P, T, x0, y0, z0, zc, QU, Bs,
                          [&](int64_t cell, int, int, int, const R qn[5], const R F[3], const R*) {
#pragma unroll
                              for (int k = 0; k < 5; ++k) qout[k * V + cell] = qn[k];
#pragma unroll
                              for (int k = 0; k < 3; ++k) Fout[k * V + cell] = F[k];
                          });
    });
}

inline size_t qforce_smem_bytes(const QTile& T, size_t real_bytes) {
    return real_bytes * (size_t)(4 * 8 * (T.tcx + 4) * (T.tcy + 4) + 3 * 16 * (T.tcx + 2) * (T.tcy + 2));
}

}  // namespace lbman
