// qpair.cuh -- FP32 Q-tensor update + body force with two points per thread
// and packed f32x2 arithmetic (sm_100: one FFMA2/FADD2/FMUL2 issue does the
// same operation on both halves of a register pair).
//
// The Q stage is bound by instruction issue, not by memory: about half of
// its instructions are FP32 arithmetic (see qforce.cuh).  Measured on B200,
// an FFMA2 stream reaches the same FMA rate as scalar FFMA (the FP32 pipe is
// not wider), but FP32 work mixed with shared-memory loads runs 1.4x faster
// packed, because each packed instruction takes one issue slot for two
// points.  This kernel is the z-marching Q+force kernel of qforce.cuh
// (same staging ring, same plane schedule, same row-stress combination)
// with every thread updating a pair of points of one row:
//   main threads : columns lbx = 1 + j and 1 + j + HP (HP = TCX / 2) of the
//                  result region, j = lane index within the row segment;
//   tail threads : the two x-halo columns 0 and TCX + 1 of a row.
// With HP = 16 a warp covers two rows, r and r + 2 (rows are visited in the
// order 0 2 1 3 4 6 5 7 ...), and the staged row length UX and the result
// row stride BXP are 8 modulo 16 words, so the two half-warps' stencil reads
// fall in disjoint banks.  Wall rules are applied to each half separately
// (they are per-point selects), so walled and periodic boxes share the code;
// warps whose points have no rule compile the rules out, as in qforce.cuh.
//
// The right-hand side is the rearranged FP32 form of physics.cuh
// (pointwise_q_mat: unhalved first differences, QB + (QB)^T co-rotation and
// alignment, N = QH products for Sigma and tau) written with explicit fused
// multiply-adds; values agree with the reference's expansion to rounding.
#pragma once

#include "physics_pair.cuh"
#include "qforce.cuh"

namespace lbman {

// ---- tile and thread geometry ----------------------------------------------
template <int TCX_, int TCY_>
struct PairTile {
    static constexpr int TCX = TCX_, TCY = TCY_;
    static_assert(TCX == 32 || TCX == 64, "pair tiles are 32 or 64 cells wide");
    static constexpr int BX = TCX + 2, BY = TCY + 2;  // halo-1 result region
    static constexpr int UY = TCY + 4;                // staged rows (halo 2)
    static constexpr int HP = TCX / 2;                // main pairs per row (16 or 32 lanes)
    static constexpr int NMAIN = HP * BY;
    static constexpr int NT = (NMAIN + BY + 31) / 32 * 32;  // main pairs, then one tail pair per row
    // result row stride: with two rows per warp (r, r + 2), 8 mod 16 words
    static constexpr int BXP = HP == 16 ? 40 : BX;
    static constexpr int NB = BXP * BY;
    template <class R>
    static constexpr size_t smem_bytes();
};

template <int TCX_, int TCY_>
template <class R>
constexpr size_t PairTile<TCX_, TCY_>::smem_bytes() {
    return Stage<PairTile<TCX_, TCY_>, R>::bytes;
}

struct PairGeo {
    int lby;                 // row in the result region
    int lbx[2];              // columns of the two points
    int p[2];                // result-plane indices lby * BXP + lbx
    int up[2];               // staged-plane indices of the two points
    int ax[2], ay;           // wrapped global coordinates
    bool has, isC[2];        // owns a pair; each point is a tile cell inside the box
    bool wx, wy, wz;         // wall rules may apply on this axis (warp-uniform after narrowing)
};

// Row of half-row h (= 2 warp + half) when two rows share a warp: rows are
// taken in the order 0 2 1 3 | 4 6 5 7 | ..., leftovers in order.
template <class TL>
__device__ __forceinline__ int pair_row(int h) {
    if constexpr (TL::HP == 32) {
        return h;
    } else {
        const int q = h >> 2, m = h & 3;
        if (4 * q + 3 >= TL::BY) return h;
        return 4 * q + ((m == 1) ? 2 : (m == 2) ? 1 : m);
    }
}

template <class TL>
__device__ __forceinline__ PairGeo pair_geo(const SimParams& P, int x0, int y0, int z0, int z1) {
    using ST = Stage<TL, float>;
    PairGeo g;
    const int t = threadIdx.x;
    const bool perx = P.qper[0] && P.qper[1] && P.uper[0] && P.uper[1];
    const bool pery = P.qper[2] && P.qper[3] && P.uper[2] && P.uper[3];
    const bool perz = P.qper[4] && P.qper[5] && P.uper[4] && P.uper[5];
    g.wx = !perx && (x0 - 1 < 1 || x0 + TL::TCX > P.nx - 2);
    g.wy = !pery && (y0 - 1 < 1 || y0 + TL::TCY > P.ny - 2);
    g.wz = !perz && (z0 - 1 < 1 || z1 > P.nz - 2);
    if (t < TL::NMAIN) {
        const int j = t % TL::HP;
        g.lby = pair_row<TL>(t / TL::HP);
        g.lbx[0] = 1 + j;
        g.lbx[1] = 1 + j + TL::HP;
        g.has = true;
    } else if (t < TL::NMAIN + TL::BY) {
        g.lby = t - TL::NMAIN;
        g.lbx[0] = 0;
        g.lbx[1] = TL::TCX + 1;
        g.has = true;
    } else {
        g.lby = 0;
        g.lbx[0] = 0;
        g.lbx[1] = 1;
        g.has = false;
    }
    g.ay = wrap_coord(y0 - 1 + g.lby, P.ny);
    const bool rowC = g.lby >= 1 && g.lby <= TL::TCY && y0 + g.lby - 1 < P.ny;
#pragma unroll
    for (int s = 0; s < 2; ++s) {
        g.p[s] = g.lby * TL::BXP + g.lbx[s];
        g.up[s] = (g.lby + 1) * ST::UX + g.lbx[s] + ST::XO - 1;
        g.ax[s] = wrap_coord(x0 - 1 + g.lbx[s], P.nx);
        g.isC[s] = g.has && rowC && g.lbx[s] >= 1 && g.lbx[s] <= TL::TCX && x0 + g.lbx[s] - 1 < P.nx;
    }
    return g;
}

// ---- wall rules on each half -------------------------------------------------
struct PairRules {
    AxisRule qx0, qx1, qy;  // both points of a pair share their row
    VRule vx0, vx1, vy;
};

// The halves are taken apart and put back by value (no reference to a
// half chosen at run time), so the pairs stay in registers.
__device__ __forceinline__ void q_apply2(const AxisRule& r0, const AxisRule& r1, const Phys<float>& K, int comp, F2 c,
                                         F2& m, F2& p) {
    float m0 = m.v.x, p0 = p.v.x, m1 = m.v.y, p1 = p.v.y;
    q_apply<float>(r0, K, comp, c.v.x, m0, p0);
    q_apply<float>(r1, K, comp, c.v.y, m1, p1);
    m = f2(m0, m1);
    p = f2(p0, p1);
}
// VelocityAxisGradient (src/boundary_handler.h:157-163) of one half, unhalved.
__device__ __forceinline__ float v_grad_half(const SimParams& P, const Phys<float>& K, const VRule& r, int comp,
                                             float m, float c, float p, bool normal) {
    if (r.m_clamp) m = c;
    if (r.p_clamp) p = c;
    if (r.m_wall) m = v_ghost<float>(P, K, r.lo, comp, c, normal);
    if (r.p_wall) p = v_ghost<float>(P, K, r.hi, comp, c, normal);
    return p - m;
}
__device__ __forceinline__ F2 v_grad2(const SimParams& P, const Phys<float>& K, const VRule& r0, const VRule& r1,
                                      int comp, F2 m, F2 c, F2 p, bool normal) {
    return f2(v_grad_half(P, K, r0, comp, m.v.x, c.v.x, p.v.x, normal),
              v_grad_half(P, K, r1, comp, m.v.y, c.v.y, p.v.y, normal));
}

__device__ __forceinline__ bool has_rule(const AxisRule& q, const VRule& v) {
    return q.m_clamp || q.p_clamp || q.m_ghost || q.p_ghost || v.m_clamp || v.p_clamp || v.m_wall || v.p_wall;
}
__device__ __forceinline__ void narrow_walls_pair(PairGeo& g, const PairRules& R) {
    const bool fx = has_rule(R.qx0, R.vx0) || has_rule(R.qx1, R.vx1);
    const bool fy = has_rule(R.qy, R.vy);
    g.wx = __any_sync(0xffffffffu, g.wx && fx);
    g.wy = __any_sync(0xffffffffu, g.wy && fy);
}

__device__ __forceinline__ F2 ld2(const float* s, int i0, int i1) { return f2(s[i0], s[i1]); }

// ---- point update of one plane ------------------------------------------------
// Results of plane zb: the row stress into the ring slots of zb, the
// Ericksen force (negated) to ern, Q_new to qn, the point's u to u.
template <class TL, bool UPWIND, int RM>
__device__ __forceinline__ void qp_compute_plane(const SimParams& P, const Phys<float>& K, const PairGeo& G,
                                                 const PairRules& R, int z0, int zb, const float* QU, float* Bs,
                                                 F2 ern[3], F2 qn[5], F2 u[3]) {
    if (!G.has) return;
    const bool rx = RM == 1 || (RM == 2 && G.wx), ry = RM == 2 && G.wy, rz = RM == 2 && G.wz;
    using ST = Stage<TL, float>;
    constexpr int NQU = ST::NQU, UX = ST::UX, NB = TL::NB;
    const float* Qc = QU + ring4(zb, z0) * 8 * NQU;
    const float* Qm = QU + ring4(zb - 1, z0) * 8 * NQU;
    const float* Qp = QU + ring4(zb + 1, z0) * 8 * NQU;
    const int u0 = G.up[0], u1 = G.up[1];
    AxisRule qz;
    VRule vz;
    if (rz) {
        const int az = wrap_coord(zb, P.nz);
        qz = q_rule(P, 2, az, P.nz);
        vz = v_rule(P, 2, az, P.nz);
    }
    F2 Q[5];
    QD2 d[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const float* qc = Qc + k * NQU;
        const F2 c = ld2(qc, u0, u1);
        F2 xm = ld2(qc, u0 - 1, u1 - 1), xp = ld2(qc, u0 + 1, u1 + 1);
        F2 ym = ld2(qc, u0 - UX, u1 - UX), yp = ld2(qc, u0 + UX, u1 + UX);
        F2 zm = ld2(Qm + k * NQU, u0, u1), zp = ld2(Qp + k * NQU, u0, u1);
        if (rx) q_apply2(R.qx0, R.qx1, K, k, c, xm, xp);
        if (ry) q_apply2(R.qy, R.qy, K, k, c, ym, yp);
        if (rz) q_apply2(qz, qz, K, k, c, zm, zp);
        d[k] = q_derivs2<UPWIND>(xm, xp, ym, yp, zm, zp, c);
        Q[k] = c;
    }
    const float* uc[3] = {Qc + 5 * NQU, Qc + 6 * NQU, Qc + 7 * NQU};
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) u[comp] = ld2(uc[comp], u0, u1);
    F2 gr[8];
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) {
        const F2 c = u[comp];
        const F2 xm = ld2(uc[comp], u0 - 1, u1 - 1), xp = ld2(uc[comp], u0 + 1, u1 + 1);
        const F2 ym = ld2(uc[comp], u0 - UX, u1 - UX), yp = ld2(uc[comp], u0 + UX, u1 + UX);
        gr[comp * 3 + 0] = rx ? v_grad2(P, K, R.vx0, R.vx1, comp, xm, c, xp, comp == 0) : xp - xm;
        gr[comp * 3 + 1] = ry ? v_grad2(P, K, R.vy, R.vy, comp, ym, c, yp, comp == 1) : yp - ym;
        if (comp < 2) {
            const F2 zm = ld2(Qm + (5 + comp) * NQU, u0, u1), zp = ld2(Qp + (5 + comp) * NQU, u0, u1);
            gr[comp * 3 + 2] = rz ? v_grad2(P, K, vz, vz, comp, zm, c, zp, false) : zp - zm;
        }
    }
    GradU2 g;
    g.ux_x = gr[0]; g.ux_y = gr[1]; g.ux_z = gr[2];
    g.uy_x = gr[3]; g.uy_y = gr[4]; g.uy_z = gr[5];
    g.uz_x = gr[6]; g.uz_y = gr[7];
    F2 pxy[6], pz[3];
    pointwise_q_pair<UPWIND>(K, Q, u[0], u[1], u[2], d, g, qn, pxy, pz, ern);
    float* Bxy = Bs + ((zb - z0) & 1) * 6 * NB;
    float* Bz = Bs + 12 * NB + ring3(zb, z0) * 3 * NB;
    const int p0 = G.p[0], p1 = G.p[1];
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        Bxy[k * NB + p0] = pxy[k].v.x;
        Bxy[k * NB + p1] = pxy[k].v.y;
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        Bz[k * NB + p0] = pz[k].v.x;
        Bz[k * NB + p1] = pz[k].v.y;
    }
}

// Body force of this thread's two tile cells in plane zc, stored by out.
template <class TL, int RM, class OutFn>
__device__ __forceinline__ void qp_force(const SimParams& P, const Phys<float>& K, const PairGeo& G,
                                         const PairRules& R, int x0, int y0, int z0, int zc, const float* Bs,
                                         const F2 ern[3], const F2 qc[5], const F2 u[3], OutFn&& out) {
    if (!(G.isC[0] || G.isC[1])) return;
    const bool rx = RM == 1 || (RM == 2 && G.wx), ry = RM == 2 && G.wy, rz = RM == 2 && G.wz;
    constexpr int NB = TL::NB, BXP = TL::BXP;
    const int p0 = G.p[0], p1 = G.p[1];
    const float* Bxy = Bs + ((zc - z0) & 1) * 6 * NB;
    const float* Bz = Bs + 12 * NB;
    const float* Bzm = Bz + ring3(zc - 1, z0) * 3 * NB;
    const float* Bzp = Bz + ring3(zc + 1, z0) * 3 * NB;
    const float* Bz0 = Bz + ring3(zc, z0) * 3 * NB;
    AxisRule qz;
    if (rz) qz = q_rule(P, 2, zc, P.nz);
    const int gy = y0 + G.lby - 1;
    F2 f[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float* px = Bxy + a * NB;
        const float* py = Bxy + (3 + a) * NB;
        F2 xm = ld2(px, p0 - 1, p1 - 1), xp = ld2(px, p0 + 1, p1 + 1);
        F2 ym = ld2(py, p0 - BXP, p1 - BXP), yp = ld2(py, p0 + BXP, p1 + BXP);
        F2 zm = ld2(Bzm + a * NB, p0, p1), zp = ld2(Bzp + a * NB, p0, p1);
        // Sigma / tau differences with the Neumann/periodic index clamp QXoff
        // (src/offsets.h:59-83, used by PassiveStressDivergence)
        if (rx) {
            const int gx0 = x0 + G.lbx[0] - 1, gx1 = x0 + G.lbx[1] - 1;
            const float c0 = px[p0], c1 = px[p1];
            float xm0 = xm.v.x, xm1 = xm.v.y, xp0 = xp.v.x, xp1 = xp.v.y;
            if (gx0 == 0 && !P.qper[0]) xm0 = c0;
            if (gx1 == 0 && !P.qper[0]) xm1 = c1;
            if (gx0 == P.nx - 1 && !P.qper[1]) xp0 = c0;
            if (gx1 == P.nx - 1 && !P.qper[1]) xp1 = c1;
            xm = f2(xm0, xm1);
            xp = f2(xp0, xp1);
        }
        if (ry) {
            const F2 c = ld2(py, p0, p1);
            if (gy == 0 && !P.qper[2]) ym = c;
            if (gy == P.ny - 1 && !P.qper[3]) yp = c;
        }
        if (rz) {
            const F2 c = ld2(Bz0 + a * NB, p0, p1);
            if (zc == 0 && !P.qper[4]) zm = c;
            if (zc == P.nz - 1 && !P.qper[5]) zp = c;
        }
        f[a] = ((xp - xm) + (yp - ym) + (zp - zm)) * f2(0.5f);
    }
    // anchoring walls: the Q_new ghost differs from the clamp (anchor_delta);
    // per point, on the halves taken apart by value
    if (rx && (R.qx0.m_ghost || R.qx0.p_ghost || R.qx1.m_ghost || R.qx1.p_ghost)) {
        const float nA = -K.ALPHA;
        f[0] = f[0] + f2(nA * anchor_delta<float>(R.qx0, K, 0, qc[0].v.x), nA * anchor_delta<float>(R.qx1, K, 0, qc[0].v.y));
        f[1] = f[1] + f2(nA * anchor_delta<float>(R.qx0, K, 1, qc[1].v.x), nA * anchor_delta<float>(R.qx1, K, 1, qc[1].v.y));
        f[2] = f[2] + f2(nA * anchor_delta<float>(R.qx0, K, 2, qc[2].v.x), nA * anchor_delta<float>(R.qx1, K, 2, qc[2].v.y));
    }
    if (ry && (R.qy.m_ghost || R.qy.p_ghost)) {
        const float nA = -K.ALPHA;
        f[0] = f[0] + f2(nA * anchor_delta<float>(R.qy, K, 1, qc[1].v.x), nA * anchor_delta<float>(R.qy, K, 1, qc[1].v.y));
        f[1] = f[1] + f2(nA * anchor_delta<float>(R.qy, K, 3, qc[3].v.x), nA * anchor_delta<float>(R.qy, K, 3, qc[3].v.y));
        f[2] = f[2] + f2(nA * anchor_delta<float>(R.qy, K, 4, qc[4].v.x), nA * anchor_delta<float>(R.qy, K, 4, qc[4].v.y));
    }
    if (rz && (qz.m_ghost || qz.p_ghost)) {
        const float nA = -K.ALPHA, A = K.ALPHA;
        f[0] = f[0] + f2(nA * anchor_delta<float>(qz, K, 2, qc[2].v.x), nA * anchor_delta<float>(qz, K, 2, qc[2].v.y));
        f[1] = f[1] + f2(nA * anchor_delta<float>(qz, K, 4, qc[4].v.x), nA * anchor_delta<float>(qz, K, 4, qc[4].v.y));
        f[2] = f[2] + f2(A * (anchor_delta<float>(qz, K, 0, qc[0].v.x) + anchor_delta<float>(qz, K, 3, qc[3].v.x)),
                         A * (anchor_delta<float>(qz, K, 0, qc[0].v.y) + anchor_delta<float>(qz, K, 3, qc[3].v.y)));
    }
    // F = Ericksen + f - MU u; ern holds the Ericksen force negated
    F2 F[3];
    const F2 nMU = f2(-K.MU);
#pragma unroll
    for (int k = 0; k < 3; ++k) F[k] = fma2(nMU, u[k], f[k]) - ern[k];
    const int64_t row = (int64_t)zc * P.nxy + (int64_t)gy * P.nx;
    if (G.isC[0]) out(row + x0 + G.lbx[0] - 1, qc[0].v.x, qc[1].v.x, qc[2].v.x, qc[3].v.x, qc[4].v.x, F[0].v.x,
                      F[1].v.x, F[2].v.x);
    if (G.isC[1]) out(row + x0 + G.lbx[1] - 1, qc[0].v.y, qc[1].v.y, qc[2].v.y, qc[3].v.y, qc[4].v.y, F[0].v.y,
                      F[1].v.y, F[2].v.y);
}

// Marches a block through planes [z0, z1) of the column at (x0, y0): the
// schedule of qf_march (qforce.cuh) with pair threads.
template <class TL, bool UPWIND, class OutFn>
__device__ __forceinline__ void qp_march(const SimParams& P, int x0, int y0, int z0, int z1,
                                         const float* __restrict__ qin, const float* __restrict__ uin, float* smem,
                                         OutFn&& out) {
    using ST = Stage<TL, float>;
    static_assert(ST::VEC, "pair tiles stage 16-byte chunks");
    float* QU = smem;
    float* Bs = smem + 4 * 8 * ST::NQU;
    const Phys<float>& K = phys_ref<float>(P);
    PairGeo G = pair_geo<TL>(P, x0, y0, z0, z1);
    PairRules R;
    R.qx0 = q_rule(P, 0, G.ax[0], P.nx);
    R.qx1 = q_rule(P, 0, G.ax[1], P.nx);
    R.vx0 = v_rule(P, 0, G.ax[0], P.nx);
    R.vx1 = v_rule(P, 0, G.ax[1], P.nx);
    R.qy = q_rule(P, 1, G.ay, P.ny);
    R.vy = v_rule(P, 1, G.ay, P.ny);
    narrow_walls_pair(G, R);
    PlaneSrc<TL, float> ps;
    plane_src_init<TL, float>(P, x0, y0, qin, uin, ps);
    F2 er_cur[3], er_next[3], qn_cur[5], qn_next[5], u_cur[3], u_next[3];

    for (int z = z0 - 2; z <= z0 + 1; ++z) qf_load_plane<TL>(P, x0, y0, z0, z, qin, uin, QU, true, ps);
    cp_async_wait_all();
    __syncthreads();
    const int rm = (G.wx || G.wy || G.wz) ? ((G.wy || G.wz) ? 2 : 1) : 0;
    // (a macro, not a lambda: passing the pair arrays to a lambda put them in
    // local memory)
#define LBMAN_QP_COMPUTE(zb, er, qn, u)                                                      \
    do {                                                                                    \
        if (rm == 0) qp_compute_plane<TL, UPWIND, 0>(P, K, G, R, z0, zb, QU, Bs, er, qn, u); \
        else if (rm == 1) qp_compute_plane<TL, UPWIND, 1>(P, K, G, R, z0, zb, QU, Bs, er, qn, u); \
        else qp_compute_plane<TL, UPWIND, 2>(P, K, G, R, z0, zb, QU, Bs, er, qn, u);         \
    } while (0)
    LBMAN_QP_COMPUTE(z0 - 1, er_next, qn_next, u_next);
    LBMAN_QP_COMPUTE(z0, er_cur, qn_cur, u_cur);
    __syncthreads();  // the slot of z0-2 is free again
    qf_load_plane<TL>(P, x0, y0, z0, z0 + 2, qin, uin, QU, true, ps);
    cp_async_wait_all();
    __syncthreads();
#pragma unroll 1
    for (int zc = z0; zc < z1; ++zc) {
        if (zc + 1 < z1) qf_load_plane<TL>(P, x0, y0, z0, zc + 3, qin, uin, QU, true, ps);
        LBMAN_QP_COMPUTE(zc + 1, er_next, qn_next, u_next);
        // no barrier here: the force of plane zc reads results of plane zc
        // written before the last barrier, in slots plane zc + 1 does not use
        if (rm == 0) qp_force<TL, 0>(P, K, G, R, x0, y0, z0, zc, Bs, er_cur, qn_cur, u_cur, out);
        else if (rm == 1) qp_force<TL, 1>(P, K, G, R, x0, y0, z0, zc, Bs, er_cur, qn_cur, u_cur, out);
        else qp_force<TL, 2>(P, K, G, R, x0, y0, z0, zc, Bs, er_cur, qn_cur, u_cur, out);
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            er_cur[k] = er_next[k];
            u_cur[k] = u_next[k];
        }
#pragma unroll
        for (int k = 0; k < 5; ++k) qn_cur[k] = qn_next[k];
        cp_async_wait_all();
        __syncthreads();
    }
#undef LBMAN_QP_COMPUTE
}

// Consumer of the split organisation: Q_new and the body force of one cell.
struct StoreQForce2 {
    float* __restrict__ qout;
    float* __restrict__ Fout;
    int64_t V;
    __device__ __forceinline__ void operator()(int64_t cell, float q0, float q1, float q2, float q3, float q4,
                                               float F0, float F1, float F2v) const {
        qout[cell] = q0;
        qout[V + cell] = q1;
        qout[2 * V + cell] = q2;
        qout[3 * V + cell] = q3;
        qout[4 * V + cell] = q4;
        Fout[cell] = F0;
        Fout[V + cell] = F1;
        Fout[2 * V + cell] = F2v;
    }
};

// The block's work: fixed z chunks or the balanced schedule (qf_run).
template <class TL, bool UPWIND, class OutFn>
__device__ __forceinline__ void qp_run(const SimParams& P, int zc_len, const float* __restrict__ qin,
                                       const float* __restrict__ uin, float* smem, OutFn&& out) {
    if (zc_len > 0) {
        const int z0 = blockIdx.z * zc_len;
        if (z0 >= P.nz) return;
        qp_march<TL, UPWIND>(P, blockIdx.x * TL::TCX, blockIdx.y * TL::TCY, z0, min(z0 + zc_len, P.nz), qin, uin,
                             smem, out);
        return;
    }
    const int cx = (P.nx + TL::TCX - 1) / TL::TCX, cy = (P.ny + TL::TCY - 1) / TL::TCY;
    const int64_t W = (int64_t)cx * cy * P.nz;
    int64_t w = W * blockIdx.x / gridDim.x;
    const int64_t w1 = W * (blockIdx.x + 1) / gridDim.x;
    while (w < w1) {
        const int64_t col = w / P.nz;
        const int z0 = (int)(w - col * P.nz);
        const int z1 = (int)min((int64_t)P.nz, z0 + (w1 - w));
        const int by = (int)(col / cx), bx = (int)(col - (int64_t)by * cx);
        qp_march<TL, UPWIND>(P, bx * TL::TCX, by * TL::TCY, z0, z1, qin, uin, smem, out);
        __syncthreads();  // the staging rings are reused by the next segment
        w += z1 - z0;
    }
}

template <class TL, bool UPWIND>
__global__ void __launch_bounds__(TL::NT, (Stage<TL, float>::MINB))
    qpair_kernel(const __grid_constant__ SimParams P, int zc_len, const float* __restrict__ qin,
                 const float* __restrict__ uin, float* __restrict__ qout, float* __restrict__ Fout) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    qp_run<TL, UPWIND>(P, zc_len, qin, uin, reinterpret_cast<float*>(smem_raw), StoreQForce2{qout, Fout, P.V});
}

}  // namespace lbman
