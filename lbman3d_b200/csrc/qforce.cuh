// qforce.cuh -- the whole Q-tensor half of a time step in one pass:
// QTensorSolver::StepAndSetupBodyForce followed by
// SetActiveStressAndComputeBodyForce (src/qtensor_solver.tpp:51-217), i.e.
// the reference's GpuQTensorStep + GpuComputeBodyForce pair
// (src/cuda/kernels.cu:122-292).
//
// Each block owns a TCX x TCY tile of the x-y plane and marches through a
// chunk of z planes.  Q and u (8 values per cell) are staged in shared memory
// as a ring of four planes with a 2-cell x-y halo, filled by cp.async one
// plane ahead; the per-point results Q_new, Sigma and tau (13 values) are kept
// as a ring of three planes with a 1-cell halo.  One thread owns one point of
// the halo tile: it computes that point's Beris-Edwards update for every
// plane, keeps its Ericksen force in registers, and -- if the point is a tile
// cell -- takes the stress divergence and grad Q_new from shared memory and
// hands the cell's Q_new, body force and u to the consumer (global stores, or
// the collide/stream of the fused kernel).  Sigma, tau, Q_new and the
// Ericksen seed never travel through HBM.
//
// Halo values are loaded with periodic wrap on every axis; the wall rules
// choose between the wrapped image, the centre value (clamp) and the
// anchoring ghost exactly as the reference's index/ghost policies do.  Blocks
// whose halo touches no wall skip the rules altogether (block-uniform test).
#pragma once

#include "physics.cuh"

namespace lbman {

template <int TCX_, int TCY_>
struct Tile {
    static constexpr int TCX = TCX_, TCY = TCY_;
    static constexpr int BX = TCX + 2, BY = TCY + 2, NB = BX * BY;  // halo-1 result region
    static constexpr int UY = TCY + 4;                               // staged rows (halo 2)
    static constexpr int NT = (NB + 31) / 32 * 32;                   // threads per block
    template <class R>
    static constexpr size_t smem_bytes();
};

// Shared-memory layout of one block for compute type R.
//   Staged Q/u: 4 planes x 8 variables x UY rows x UX columns.  FP32 tiles
//   whose width is a multiple of 4 stage x in [x0-4, x0+TCX+4) as 16-byte
//   chunks; otherwise x in [x0-2, x0+TCX+2) one value per copy.
//   Results: FP64 keeps Q_new, Sigma and tau (13 values) for 3 planes and
//   differentiates each along every axis, in the reference's order.  FP32
//   keeps the row stress Pi = Sigma + tau - ALPHA Q_new pre-combined per
//   differentiation axis: 6 values (the x- and y-differenced rows) for the
//   current and next plane, 3 values (the z-differenced row) for 3 planes.
template <class TL, class R>
struct Stage {
    static constexpr bool VEC = sizeof(R) == 4 && TL::TCX % 4 == 0;
    static constexpr bool COMB = sizeof(R) == 4;
    static constexpr int XO = VEC ? 4 : 2;        // staged column of global x0
    static constexpr int UX = TL::TCX + 2 * XO;   // staged row length
    static constexpr int NQU = UX * TL::UY;       // one variable of one plane
    static constexpr int NRES = COMB ? (2 * 6 + 3 * 3) : 3 * 13;
    static constexpr size_t bytes = sizeof(R) * (size_t)(4 * 8 * NQU + NRES * TL::NB);
    // Blocks per SM that the shared memory admits (228 KB per SM, 1 KB
    // reserved per block); the Q+force kernel caps its registers to match.
    static constexpr int FIT = (int)((228 * 1024) / (bytes + 1024));
    static constexpr int MINB = FIT < 1 ? 1 : (FIT > 4 ? 4 : FIT);
};

template <int TCX_, int TCY_>
template <class R>
constexpr size_t Tile<TCX_, TCY_>::smem_bytes() {
    return Stage<Tile<TCX_, TCY_>, R>::bytes;
}

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
__device__ __forceinline__ void cp_async16(float* s, const float* g) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"((unsigned)__cvta_generic_to_shared(s)),
                 "l"(g));
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// Source addresses of the 16-byte chunks (FP32 vec staging) that this
// thread copies for every plane -- tile + 2-cell halo, all 8 variables --
// without the plane offset.  Set once per column segment, so each plane's
// copies cost one address add apiece.  Chunk k of thread t is chunk
// i = t + k NT of the plane; its shared-memory offset within the plane slot
// is 4 i (row-major rows of UX = 4 CH values).
template <class TL, class R>
struct PlaneSrc {
    using ST = Stage<TL, R>;
    static constexpr int CH = ST::UX / 4;
    static constexpr int N = 8 * TL::UY * CH;
    static constexpr int NCH = ST::VEC ? (N + TL::NT - 1) / TL::NT : 1;
    const R* src[NCH];
};

template <class TL, class R>
__device__ __forceinline__ void plane_src_init(const SimParams& P, int x0, int y0, const R* __restrict__ qin,
                                               const R* __restrict__ uin, PlaneSrc<TL, R>& ps) {
    using PS = PlaneSrc<TL, R>;
    if constexpr (Stage<TL, R>::VEC) {
#pragma unroll
        for (int k = 0; k < PS::NCH; ++k) {
            const int i = threadIdx.x + k * TL::NT;
            if (i >= PS::N) {
                ps.src[k] = qin;
                continue;
            }
            const int row = i / PS::CH, ch = i - row * PS::CH;
            const int var = row / TL::UY, ly = row - var * TL::UY;
            const int gy = wrap_coord(y0 - 2 + ly, P.ny);
            const int gx = wrap_coord(x0 - Stage<TL, R>::XO + 4 * ch, P.nx);
            ps.src[k] = (var < 5 ? qin + (int64_t)var * P.V : uin + (int64_t)(var - 5) * P.V) +
                        (int64_t)gy * P.nx + gx;
        }
    }
}

// Issue the copies of plane zg (Q then u, tile + 2-cell halo, periodic wrap)
// into its ring slot; complete at the next cp_async_wait_all().  vec: 16-byte
// chunks from the precomputed sources (FP32, nx a multiple of 4, 16-byte
// aligned fields), so no chunk straddles the periodic seam.
template <class TL, class R>
__device__ __forceinline__ void qf_load_plane(const SimParams& P, int x0, int y0, int z0, int zg,
                                              const R* __restrict__ qin, const R* __restrict__ uin, R* QU,
                                              bool vec, const PlaneSrc<TL, R>& ps) {
    using ST = Stage<TL, R>;
    const int zw = wrap_coord(zg, P.nz);
    R* dst = QU + ring4(zg, z0) * 8 * ST::NQU;
    const int64_t zoff = (int64_t)zw * P.nxy;
    if constexpr (ST::VEC) {
        if (vec) {
            using PS = PlaneSrc<TL, R>;
            R* d = dst + 4 * threadIdx.x;
#pragma unroll
            for (int k = 0; k < PS::NCH; ++k) {
                if ((k + 1) * TL::NT <= PS::N || threadIdx.x + k * TL::NT < PS::N)
                    cp_async16(d + 4 * k * TL::NT, ps.src[k] + zoff);
            }
            return;
        }
    }
    constexpr int N = 8 * TL::UY * ST::UX;
#pragma unroll 1
    for (int i = threadIdx.x; i < N; i += TL::NT) {
        const int row = i / ST::UX, lx = i - row * ST::UX;
        const int var = row / TL::UY, ly = row - var * TL::UY;
        const int gy = wrap_coord(y0 - 2 + ly, P.ny);
        const int gx = wrap_coord(x0 - ST::XO + lx, P.nx);
        const R* src = (var < 5 ? qin + (int64_t)var * P.V : uin + (int64_t)(var - 5) * P.V) + zoff +
                       (int64_t)gy * P.nx + gx;
        cp_async(dst + var * ST::NQU + ly * ST::UX + lx, src);
    }
}

// Per-thread geometry, fixed for the whole z march.
struct PointGeo {
    int lbx, lby;     // position in the result region
    int p;            // its index in the result planes, lby * BX + lbx
    int ax, ay;       // wrapped global coordinates of the point
    bool hasB, isC;   // owns a result point / a tile cell
    bool wx, wy, wz;  // wall rules may apply on this axis: wz block-uniform,
                      // wx / wy warp-uniform (see narrow_walls)
};

template <class TL>
__device__ __forceinline__ PointGeo point_geo(const SimParams& P, int x0, int y0, int z0, int z1) {
    PointGeo g;
    const int t = threadIdx.x;
    const bool perx = P.qper[0] && P.qper[1] && P.uper[0] && P.uper[1];
    const bool pery = P.qper[2] && P.qper[3] && P.uper[2] && P.uper[3];
    const bool perz = P.qper[4] && P.qper[5] && P.uper[4] && P.uper[5];
    g.wx = !perx && (x0 - 1 < 1 || x0 + TL::TCX > P.nx - 2);
    g.wy = !pery && (y0 - 1 < 1 || y0 + TL::TCY > P.ny - 2);
    g.wz = !perz && (z0 - 1 < 1 || z1 > P.nz - 2);
    g.hasB = t < TL::NB;
    if constexpr (TL::BX >= 32) {
        // Whole warps take 32-point row segments, so the stencil reads of a
        // warp fall on consecutive shared-memory words (no bank conflicts);
        // the last warp(s) take the TAIL leftover columns of every row.  In a
        // block on the x-low wall the segments start at column 2, so the two
        // wall-side columns (the wall point and the halo point beyond it)
        // fall in the tail warp, as the x-high wall's columns already do.
        constexpr int WPR = TL::BX / 32, NW = WPR * TL::BY, TAIL = TL::BX - 32 * WPR;
        const int s = (TAIL >= 2 && g.wx && x0 == 0) ? 2 : 0;
        const int w = t >> 5;
        if (w < NW) {
            g.lby = w / WPR;
            g.lbx = s + (w - g.lby * WPR) * 32 + (t & 31);
        } else if constexpr (TAIL > 0) {
            const int k = t - 32 * NW;
            g.lby = k / TAIL;
            const int j = k - g.lby * TAIL;
            g.lbx = j < s ? j : j + 32 * WPR;
        } else {
            g.lby = TL::BY;
            g.lbx = 0;
        }
    } else {
        g.lbx = t % TL::BX;
        g.lby = t / TL::BX;
    }
    g.p = g.lby * TL::BX + g.lbx;
    g.ax = wrap_coord(x0 - 1 + g.lbx, P.nx);
    g.ay = wrap_coord(y0 - 1 + g.lby, P.ny);
    g.isC = g.hasB && g.lbx >= 1 && g.lbx <= TL::TCX && g.lby >= 1 && g.lby <= TL::TCY &&
            x0 + g.lbx - 1 < P.nx && y0 + g.lby - 1 < P.ny;
    return g;
}

// Narrows the block-uniform wx / wy to the warps that hold a point with a
// wall rule on that axis (any clamp, ghost or wall flag of its Q or velocity
// rule), so the other warps of a wall block skip the rule code.
__device__ __forceinline__ void narrow_walls(PointGeo& g, const AxisRule& qx, const AxisRule& qy,
                                             const VRule& vx, const VRule& vy) {
    const bool fx = g.wx && (qx.m_clamp || qx.p_clamp || qx.m_ghost || qx.p_ghost || vx.m_clamp || vx.p_clamp ||
                             vx.m_wall || vx.p_wall);
    const bool fy = g.wy && (qy.m_clamp || qy.p_clamp || qy.m_ghost || qy.p_ghost || vy.m_clamp || vy.p_clamp ||
                             vy.m_wall || vy.p_wall);
    g.wx = __any_sync(0xffffffffu, fx);
    g.wy = __any_sync(0xffffffffu, fy);
}

// Beris-Edwards update of this thread's point in plane zb; results to the
// ring slots of zb, Ericksen force to er, Q_new to qn.
// RM: which wall-rule code is compiled in -- 0 none, 1 the x axis only
// (every point's y and z rules are off), 2 all axes as the flags say.
template <class TL, class R, bool UPWIND, int RM>
__device__ __forceinline__ void qf_compute_plane(const SimParams& P, const Phys<R>& K, const PointGeo& G,
                                                 const AxisRule& qx, const AxisRule& qy, const VRule& vx,
                                                 const VRule& vy, int z0, int zb, const R* QU, R* Bs,
                                                 R er[3], R qn[5]) {
    if (!G.hasB) return;
    // wall rules compiled in and active in this warp, per axis
    const bool rx = RM == 1 || (RM == 2 && G.wx), ry = RM == 2 && G.wy, rz = RM == 2 && G.wz;
    using ST = Stage<TL, R>;
    constexpr int NQU = ST::NQU, UX = ST::UX, NB = TL::NB;
    const R* Qc = QU + ring4(zb, z0) * 8 * NQU;
    const R* Qm = QU + ring4(zb - 1, z0) * 8 * NQU;
    const R* Qp = QU + ring4(zb + 1, z0) * 8 * NQU;
    const int up = (G.lby + 1) * UX + G.lbx + ST::XO - 1;
    AxisRule qz;
    VRule vz;
    if (rz) {
        const int az = wrap_coord(zb, P.nz);
        qz = q_rule(P, 2, az, P.nz);
        vz = v_rule(P, 2, az, P.nz);
    }
    R Q[5];
    QD<R> d[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const R* qc = Qc + k * NQU;
        const R c = qc[up];
        R xm = qc[up - 1], xp = qc[up + 1], ym = qc[up - UX], yp = qc[up + UX];
        R zm = Qm[k * NQU + up], zp = Qp[k * NQU + up];
        if (rx) q_apply<R>(qx, K, k, c, xm, xp);
        if (ry) q_apply<R>(qy, K, k, c, ym, yp);
        if (rz) q_apply<R>(qz, K, k, c, zm, zp);
        d[k] = q_derivs<R, !ST::COMB>(xm, xp, ym, yp, zm, zp, c);
        Q[k] = c;
    }
    const R* uc[3] = {Qc + 5 * NQU, Qc + 6 * NQU, Qc + 7 * NQU};
    const R u0[3] = {uc[0][up], uc[1][up], uc[2][up]};
    // (component, axis) pairs of the stored gradient: ux_x ux_y ux_z uy_x uy_y uy_z uz_x uz_y
    // FP32 (COMB) keeps the differences unhalved; pointwise_q_mat folds the 1/2.
    constexpr R HS = ST::COMB ? R(1.0) : R(0.5);
    R gr[8];
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) {
        const R c = u0[comp];
        const R xm = uc[comp][up - 1], xp = uc[comp][up + 1];
        const R ym = uc[comp][up - UX], yp = uc[comp][up + UX];
        gr[comp * 3 + 0] = rx ? v_grad<R, !ST::COMB>(P, K, vx, comp, xm, c, xp, comp == 0) : HS * (xp - xm);
        gr[comp * 3 + 1] = ry ? v_grad<R, !ST::COMB>(P, K, vy, comp, ym, c, yp, comp == 1) : HS * (yp - ym);
        if (comp < 2) {
            const R zm = Qm[(5 + comp) * NQU + up], zp = Qp[(5 + comp) * NQU + up];
            gr[comp * 3 + 2] = rz ? v_grad<R, !ST::COMB>(P, K, vz, comp, zm, c, zp, false) : HS * (zp - zm);
        }
    }
    GradU<R> g;
    g.ux_x = gr[0]; g.ux_y = gr[1]; g.ux_z = gr[2];
    g.uy_x = gr[3]; g.uy_y = gr[4]; g.uy_z = gr[5];
    g.uz_x = gr[6]; g.uz_y = gr[7];
    R sg[5], ta[3];
    if constexpr (ST::COMB)
        pointwise_q_mat<R, UPWIND>(K, Q, u0[0], u0[1], u0[2], d, g, qn, sg, ta, er);
    else
        pointwise_q<R, UPWIND>(K, Q, u0[0], u0[1], u0[2], d, g, qn, sg, ta, er);
    if constexpr (ST::COMB) {
        // Row stress Pi_ab = Sigma_ab + tau_ab - ALPHA Q_new_ab (tau_ba = -tau_ab),
        // grouped by the axis b it is differentiated along (f_a = d_b Pi_ab).
        const R a = -K.ALPHA;
        R* Bxy = Bs + ((zb - z0) & 1) * 6 * NB + G.p;
        R* Bz = Bs + 12 * NB + ring3(zb, z0) * 3 * NB + G.p;
        Bxy[0 * NB] = sg[0] + a * qn[0];
        Bxy[1 * NB] = (sg[1] - ta[0]) + a * qn[1];
        Bxy[2 * NB] = (sg[2] - ta[1]) + a * qn[2];
        Bxy[3 * NB] = (sg[1] + ta[0]) + a * qn[1];
        Bxy[4 * NB] = sg[3] + a * qn[3];
        Bxy[5 * NB] = (sg[4] - ta[2]) + a * qn[4];
        Bz[0 * NB] = (sg[2] + ta[1]) + a * qn[2];
        Bz[1 * NB] = (sg[4] + ta[2]) + a * qn[4];
        Bz[2 * NB] = -(sg[0] + sg[3]) - a * (qn[0] + qn[3]);
    } else {
        R* Bd = Bs + ring3(zb, z0) * 13 * NB + G.p;
#pragma unroll
        for (int k = 0; k < 5; ++k) Bd[k * NB] = qn[k];
#pragma unroll
        for (int k = 0; k < 5; ++k) Bd[(5 + k) * NB] = sg[k];
#pragma unroll
        for (int k = 0; k < 3; ++k) Bd[(10 + k) * NB] = ta[k];
    }
}

// Difference of the active term's Q_new derivative between the anchoring
// ghost and the index clamp, at a wall cell: the clamp takes the centre c
// for the missing neighbour, the ghost 2A - c (QAxisGhostPair,
// src/boundary_handler.h:253-282), so d_ghost - d_clamp = c - A_lo at the
// low face and A_hi - c at the high face.
template <class R>
__device__ __forceinline__ R anchor_delta(const AxisRule& r, const Phys<R>& K, int k, R c) {
    R d = R(0);
    if (r.m_ghost) d += c - K.anchor[r.lo][k];
    if (r.p_ghost) d += K.anchor[r.hi][k] - c;
    return d;
}

// Body force of this thread's tile cell in plane zc from the staged result
// planes; out(cell, x, y, z, qn[5], F[3], u[3]) consumes it.  qc is the
// cell's Q_new (kept in registers by the FP32 path).
template <class TL, class R, int RM, class OutFn>
__device__ __forceinline__ void qf_force_cell(const SimParams& P, const Phys<R>& K, const PointGeo& G,
                                              const AxisRule& qx, const AxisRule& qy, int x0, int y0, int z0,
                                              int zc, const R* QU, const R* Bs, const R er[3], const R qc[5],
                                              OutFn&& out) {
    if (!G.isC) return;
    // wall rules compiled in and active in this warp, per axis
    const bool rx = RM == 1 || (RM == 2 && G.wx), ry = RM == 2 && G.wy, rz = RM == 2 && G.wz;
    using ST = Stage<TL, R>;
    constexpr int NB = TL::NB, BX = TL::BX;
    const int t = G.p;
    const int gx = x0 + G.lbx - 1, gy = y0 + G.lby - 1;
    AxisRule qz;
    if (rz) qz = q_rule(P, 2, zc, P.nz);
    // Sigma / tau differences with the Neumann/periodic index clamp QXoff
    // (src/offsets.h:59-83, used by PassiveStressDivergence).
    const bool xmc = rx && gx == 0 && !P.qper[0], xpc = rx && gx == P.nx - 1 && !P.qper[1];
    const bool ymc = ry && gy == 0 && !P.qper[2], ypc = ry && gy == P.ny - 1 && !P.qper[3];
    const bool zmc = rz && zc == 0 && !P.qper[4], zpc = rz && zc == P.nz - 1 && !P.qper[5];
    const R* U0 = QU + ring4(zc, z0) * 8 * ST::NQU;
    const int up = (G.lby + 1) * ST::UX + G.lbx + ST::XO - 1;
    const R u[3] = {U0[5 * ST::NQU + up], U0[6 * ST::NQU + up], U0[7 * ST::NQU + up]};
    R F[3];
    if constexpr (ST::COMB) {
        const R* Bxy = Bs + ((zc - z0) & 1) * 6 * NB + t;
        const R* Bz = Bs + 12 * NB + t;
        const R* Bzm = Bz + ring3(zc - 1, z0) * 3 * NB;
        const R* Bzp = Bz + ring3(zc + 1, z0) * 3 * NB;
        const R* Bz0 = Bz + ring3(zc, z0) * 3 * NB;
        R f[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            const R* px = Bxy + a * NB;
            const R* py = Bxy + (3 + a) * NB;
            R xm = px[-1], xp = px[1], ym = py[-BX], yp = py[BX];
            R zm = Bzm[a * NB], zp = Bzp[a * NB];
            if (rx) {
                if (xmc) xm = px[0];
                if (xpc) xp = px[0];
            }
            if (ry) {
                if (ymc) ym = py[0];
                if (ypc) yp = py[0];
            }
            if (rz) {
                if (zmc) zm = Bz0[a * NB];
                if (zpc) zp = Bz0[a * NB];
            }
            f[a] = R(0.5) * (xp - xm) + R(0.5) * (yp - ym) + R(0.5) * (zp - zm);
        }
        if (rx && (qx.m_ghost || qx.p_ghost)) {
            f[0] += -K.ALPHA * anchor_delta<R>(qx, K, 0, qc[0]);
            f[1] += -K.ALPHA * anchor_delta<R>(qx, K, 1, qc[1]);
            f[2] += -K.ALPHA * anchor_delta<R>(qx, K, 2, qc[2]);
        }
        if (ry && (qy.m_ghost || qy.p_ghost)) {
            f[0] += -K.ALPHA * anchor_delta<R>(qy, K, 1, qc[1]);
            f[1] += -K.ALPHA * anchor_delta<R>(qy, K, 3, qc[3]);
            f[2] += -K.ALPHA * anchor_delta<R>(qy, K, 4, qc[4]);
        }
        if (rz && (qz.m_ghost || qz.p_ghost)) {
            f[0] += -K.ALPHA * anchor_delta<R>(qz, K, 2, qc[2]);
            f[1] += -K.ALPHA * anchor_delta<R>(qz, K, 4, qc[4]);
            f[2] += K.ALPHA * (anchor_delta<R>(qz, K, 0, qc[0]) + anchor_delta<R>(qz, K, 3, qc[3]));
        }
        F[0] = er[0] + (f[0] - K.MU * u[0]);
        F[1] = er[1] + (f[1] - K.MU * u[1]);
        F[2] = er[2] + (f[2] - K.MU * u[2]);
        const int64_t cell = (int64_t)zc * P.nxy + (int64_t)gy * P.nx + gx;
        out(cell, gx, gy, zc, qc, F, u);
    } else {
        const R* B0 = Bs + ring3(zc, z0) * 13 * NB;
        const R* Bm = Bs + ring3(zc - 1, z0) * 13 * NB;
        const R* Bp = Bs + ring3(zc + 1, z0) * 13 * NB;
        // grad Q_new with the wall ghosts (QGradientAndLaplacian on the new Q)
        R dQ[5][3], qn[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            const R* b = B0 + k * NB;
            const R c = b[t];
            qn[k] = c;
            R xm = b[t - 1], xp = b[t + 1], ym = b[t - BX], yp = b[t + BX];
            R zm = Bm[k * NB + t], zp = Bp[k * NB + t];
            if (rx) q_apply<R>(qx, K, k, c, xm, xp);
            if (ry) q_apply<R>(qy, K, k, c, ym, yp);
            if (rz) q_apply<R>(qz, K, k, c, zm, zp);
            dQ[k][0] = R(0.5) * (xp - xm);
            dQ[k][1] = R(0.5) * (yp - ym);
            dQ[k][2] = R(0.5) * (zp - zm);
        }
        R dS[3][5], dT[3][3];
#pragma unroll
        for (int v = 0; v < 8; ++v) {
            const R* b = B0 + (5 + v) * NB;
            const R c = b[t];
            const R xm = xmc ? c : b[t - 1], xp = xpc ? c : b[t + 1];
            const R ym = ymc ? c : b[t - BX], yp = ypc ? c : b[t + BX];
            const R zm = zmc ? c : Bm[(5 + v) * NB + t], zp = zpc ? c : Bp[(5 + v) * NB + t];
            const R ddx = R(0.5) * (xp - xm), ddy = R(0.5) * (yp - ym), ddz = R(0.5) * (zp - zm);
            if (v < 5) { dS[0][v] = ddx; dS[1][v] = ddy; dS[2][v] = ddz; }
            else { dT[0][v - 5] = ddx; dT[1][v - 5] = ddy; dT[2][v - 5] = ddz; }
        }
        active_passive_force<R>(K, dQ, dS, dT, u[0], u[1], u[2], er, F);
        const int64_t cell = (int64_t)zc * P.nxy + (int64_t)gy * P.nx + gx;
        out(cell, gx, gy, zc, qn, F, u);
    }
}

// Marches a block through planes [z0, z1) of the column at (x0, y0).  The
// copy of plane zc+3 is in flight while planes zc+1 (results) and zc (force,
// consumer) are computed.
template <class TL, class R, bool UPWIND, class OutFn>
__device__ __forceinline__ void qf_march(const SimParams& P, int x0, int y0, int z0, int z1,
                                         const R* __restrict__ qin, const R* __restrict__ uin, R* smem,
                                         OutFn&& out) {
    using ST = Stage<TL, R>;
    R* QU = smem;
    R* Bs = smem + 4 * 8 * ST::NQU;
    const Phys<R>& K = phys_ref<R>(P);
    PointGeo G = point_geo<TL>(P, x0, y0, z0, z1);
    const AxisRule qx = q_rule(P, 0, G.ax, P.nx), qy = q_rule(P, 1, G.ay, P.ny);
    const VRule vx = v_rule(P, 0, G.ax, P.nx), vy = v_rule(P, 1, G.ay, P.ny);
    narrow_walls(G, qx, qy, vx, vy);
    const bool vec = ST::VEC && (P.nx & 3) == 0 &&
                     ((reinterpret_cast<uintptr_t>(qin) | reinterpret_cast<uintptr_t>(uin)) & 15) == 0;
    R er_cur[3], er_next[3], qn_cur[5], qn_next[5];
    PlaneSrc<TL, R> ps;
    if (vec) plane_src_init<TL, R>(P, x0, y0, qin, uin, ps);

    for (int z = z0 - 2; z <= z0 + 1; ++z) qf_load_plane<TL>(P, x0, y0, z0, z, qin, uin, QU, vec, ps);
    cp_async_wait_all();
    __syncthreads();
    // Warps none of whose points has a wall rule run the point update and
    // the force with the rule code compiled out, warps with x rules only
    // (the slit's wall columns) a copy without the y and z rule code; one
    // warp-uniform choice per warp, made once per column segment.
    const int rm = (G.wx || G.wy || G.wz) ? ((G.wy || G.wz) ? 2 : 1) : 0;
    auto compute = [&](int zb, R er[3], R qn[5]) {
        if (rm == 0) qf_compute_plane<TL, R, UPWIND, 0>(P, K, G, qx, qy, vx, vy, z0, zb, QU, Bs, er, qn);
        else if (rm == 1) qf_compute_plane<TL, R, UPWIND, 1>(P, K, G, qx, qy, vx, vy, z0, zb, QU, Bs, er, qn);
        else qf_compute_plane<TL, R, UPWIND, 2>(P, K, G, qx, qy, vx, vy, z0, zb, QU, Bs, er, qn);
    };
    compute(z0 - 1, er_next, qn_next);
    compute(z0, er_cur, qn_cur);
    __syncthreads();  // the slot of z0-2 is free again
    qf_load_plane<TL>(P, x0, y0, z0, z0 + 2, qin, uin, QU, vec, ps);
    cp_async_wait_all();
    __syncthreads();
#pragma unroll 1
    for (int zc = z0; zc < z1; ++zc) {
        if (zc + 1 < z1) qf_load_plane<TL>(P, x0, y0, z0, zc + 3, qin, uin, QU, vec, ps);
        compute(zc + 1, er_next, qn_next);
        // No barrier here: the force of plane zc reads its neighbours' results
        // of plane zc (written before the last barrier, in a slot that plane
        // zc + 1 does not use) and the z-ring only at its own point.
        if (rm == 0) qf_force_cell<TL, R, 0>(P, K, G, qx, qy, x0, y0, z0, zc, QU, Bs, er_cur, qn_cur, out);
        else if (rm == 1) qf_force_cell<TL, R, 1>(P, K, G, qx, qy, x0, y0, z0, zc, QU, Bs, er_cur, qn_cur, out);
        else qf_force_cell<TL, R, 2>(P, K, G, qx, qy, x0, y0, z0, zc, QU, Bs, er_cur, qn_cur, out);
#pragma unroll
        for (int k = 0; k < 3; ++k) er_cur[k] = er_next[k];
#pragma unroll
        for (int k = 0; k < 5; ++k) qn_cur[k] = qn_next[k];
        cp_async_wait_all();
        __syncthreads();
    }
}

// Work of one block of a single-box launch.  zc_len > 0: block (bx, by, bz)
// marches z chunk bz of column (bx, by).  zc_len <= 0 (balanced): the grid is
// a whole number of waves of resident blocks, and block b takes the b-th
// equal share of the column-major sequence of (column, plane) units -- one
// or two partial columns -- so blocks finish within a plane of each other
// and no partial last wave idles the SMs.
template <class TL, class R, bool UPWIND, class OutFn>
__device__ __forceinline__ void qf_run(const SimParams& P, int zc_len, const R* __restrict__ qin,
                                       const R* __restrict__ uin, R* smem, OutFn&& out) {
    if (zc_len > 0) {
        const int z0 = P.zlo + (int)blockIdx.z * zc_len;
        if (z0 >= P.zhi) return;
        qf_march<TL, R, UPWIND>(P, blockIdx.x * TL::TCX, blockIdx.y * TL::TCY, z0, min(z0 + zc_len, P.zhi), qin,
                                uin, smem, out);
        return;
    }
    const int cx = (P.nx + TL::TCX - 1) / TL::TCX, cy = (P.ny + TL::TCY - 1) / TL::TCY;
    const int nzo = P.zhi - P.zlo;
    const int64_t W = (int64_t)cx * cy * nzo;
    int64_t w = W * blockIdx.x / gridDim.x;
    const int64_t w1 = W * (blockIdx.x + 1) / gridDim.x;
    while (w < w1) {
        const int64_t col = w / nzo;
        const int z0 = P.zlo + (int)(w - col * nzo);
        const int z1 = (int)min((int64_t)P.zhi, z0 + (w1 - w));
        const int by = (int)(col / cx), bx = (int)(col - (int64_t)by * cx);
        qf_march<TL, R, UPWIND>(P, bx * TL::TCX, by * TL::TCY, z0, z1, qin, uin, smem, out);
        __syncthreads();  // the staging rings are reused by the next segment
        w += z1 - z0;
    }
}

// Consumer of the split organisation: store Q_new and the body force.
template <class R>
struct StoreQForce {
    R* __restrict__ qout;
    R* __restrict__ Fout;
    int64_t V;
    __device__ __forceinline__ void operator()(int64_t cell, int, int, int, const R qn[5], const R F[3],
                                               const R*) const {
#pragma unroll
        for (int k = 0; k < 5; ++k) qout[k * V + cell] = qn[k];
#pragma unroll
        for (int k = 0; k < 3; ++k) Fout[k * V + cell] = F[k];
    }
};

template <class TL, class R, bool UPWIND>
__global__ void __launch_bounds__(TL::NT, (Stage<TL, R>::MINB)) qforce_kernel(const __grid_constant__ SimParams P, int zc_len,
                                                        const R* __restrict__ qin, const R* __restrict__ uin,
                                                        R* __restrict__ qout, R* __restrict__ Fout) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    qf_run<TL, R, UPWIND>(P, zc_len, qin, uin, reinterpret_cast<R*>(smem_raw), StoreQForce<R>{qout, Fout, P.V});
}

}  // namespace lbman
