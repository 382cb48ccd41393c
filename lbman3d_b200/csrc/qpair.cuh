// qpair.cuh -- FP32 Q-tensor update + body force with two points per thread
// and packed f32x2 arithmetic (sm_100: one FFMA2/FADD2/FMUL2 issue does the
// same operation on both halves of a register pair).
//
// The Q stage is bound by instruction issue, not by memory: about half of
// its instructions are FP32 arithmetic (see qforce.cuh).  Measured on B200,
// an FFMA2 stream reaches the same FMA rate as scalar FFMA (the FP32 pipe is
// not wider), but FP32 work mixed with shared-memory loads runs 1.4x faster
// packed, because each packed instruction takes one issue slot for two
// points.  This kernel marches z like qforce.cuh (cp.async staging ring of
// Q and u, one barrier per plane, row stress of the FP32 form) with these
// differences:
//   * a tile is 30 cells wide, so a row of the halo-1 result region is 32
//     points: thread j of a row updates the pair (j, j + 16); a warp takes
//     two rows r and r + 2 (rows in the order 0 2 1 3 | 4 6 5 7 | ...; the
//     tile heights make the row count a multiple of 4).  The staged row
//     length and the result row stride are 40 words (8 mod 16), so the two
//     half-warps' reads fall in disjoint banks.  The staging window starts at
//     the 16-byte boundary at or below x0 - 2 and is 36 columns wide;
//   * the z derivative of the row stress reads only the thread's own column,
//     so its three planes live in registers, not shared memory, and the
//     force of plane zc is accumulated before plane zc + 1 is updated (all
//     but the +z term), which ends the life of that plane's Q_new, u and
//     Ericksen force before the next update starts;
//   * where shared memory allows it without losing a block per SM, the
//     staging ring holds five planes and each copy gets two planes of lead.
// Wall rules are applied to each half separately (they are per-point
// selects); warps whose points have no rule compile them out.
#pragma once

#include "physics_pair.cuh"
#include "qforce.cuh"

namespace lbman {

// ---- tile and shared-memory geometry -----------------------------------------
template <int TCX_, int TCY_>
struct PairTile {
    static constexpr int TCX = TCX_, TCY = TCY_;
    static_assert(TCX == 30, "a pair tile is 30 cells wide: 32 result points per row");
    static constexpr int BX = TCX + 2, BY = TCY + 2;  // halo-1 result region
    static_assert(BY % 4 == 0, "rows are paired (r, r + 2) in groups of four");
    static constexpr int UY = TCY + 4;                // staged rows (halo 2)
    static constexpr int HP = BX / 2;                 // 16 pairs per row
    static constexpr int NT = HP * BY;                // threads: one per pair
    static constexpr int UX = 40;                     // staged row length (36 used)
    static constexpr int CH = 9;                      // 16-byte chunks per staged row
    static constexpr int NQU = UX * UY;               // one variable of one plane
    static constexpr int BXP = 40;                    // result row stride
    static constexpr int NB = BXP * BY;
    static constexpr size_t result_floats = (size_t)2 * 6 * NB;   // 2 planes x row stress (x, y)
    // Blocks per SM that shared memory admits (228 KB per SM, 1 KB reserved
    // per block) with an ns-plane staging ring of Q (5) and u (3).
    static constexpr int fit(int ns) {
        return (int)((228 * 1024) / (sizeof(float) * ((size_t)ns * 8 * NQU + result_floats) + 1024));
    }
    // Staging ring: 3 planes being read plus the copies in flight.  Five
    // planes (two copies in flight) where that keeps the blocks per SM of a
    // four-plane ring, else four.
    static constexpr int NS = fit(5) == fit(4) ? 5 : 4;
    static constexpr int LEAD = NS - 3;                           // planes copied ahead
    static constexpr size_t stage_floats = (size_t)NS * 8 * NQU;
    template <class R>
    static constexpr size_t smem_bytes() {
        return sizeof(float) * (stage_floats + result_floats);
    }
    static constexpr int FIT = fit(NS);
    static constexpr int MINB = FIT < 1 ? 1 : (FIT > 3 ? 3 : FIT);
    // chunks per plane and per thread
    static constexpr int NCHUNK = 8 * UY * CH;
    static constexpr int NCH = (NCHUNK + NT - 1) / NT;
};

// Global sources of this thread's staging chunks, without the plane offset;
// chunk i = t + k NT of a plane goes to row i / CH, column 4 (i % CH).
template <class TL>
struct PairSrc {
    const float* src[TL::NCH];
};

template <class TL>
__device__ __forceinline__ void pair_src_init(const SimParams& P, int s0, int y0, const float* __restrict__ qin,
                                              const float* __restrict__ uin, PairSrc<TL>& ps) {
#pragma unroll
    for (int k = 0; k < TL::NCH; ++k) {
        const int i = threadIdx.x + k * TL::NT;
        if (i >= TL::NCHUNK) {
            ps.src[k] = qin;
            continue;
        }
        const int row = i / TL::CH, ch = i - row * TL::CH;
        const int var = row / TL::UY, ly = row - var * TL::UY;
        const int gy = wrap_coord(y0 - 2 + ly, P.ny);
        const int gx = wrap_coord(s0 + 4 * ch, P.nx);  // nx % 4 == 0: no chunk straddles the seam
        ps.src[k] = (var < 5 ? qin + (int64_t)var * P.V : uin + (int64_t)(var - 5) * P.V) + (int64_t)gy * P.nx + gx;
    }
}

// Ring slot of staged plane z of a march starting at z0 (z >= z0 - 2).
template <class TL>
__device__ __forceinline__ int pair_slot(int z, int z0) {
    return (z - z0 + 2) % TL::NS;
}

__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait_group() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

// Issues the copies of plane zg (one commit group per plane, issued by the
// caller after the call).
template <class TL>
__device__ __forceinline__ void pair_load_plane(const SimParams& P, int z0, int zg, float* QU, const PairSrc<TL>& ps) {
    const int zw = wrap_coord(zg, P.nz);
    float* dst = QU + pair_slot<TL>(zg, z0) * 8 * TL::NQU;
    const int64_t zoff = (int64_t)zw * P.nxy;
#pragma unroll
    for (int k = 0; k < TL::NCH; ++k) {
        const int i = threadIdx.x + k * TL::NT;
        if ((k + 1) * TL::NT <= TL::NCHUNK || i < TL::NCHUNK) {
            const int row = i / TL::CH, ch = i - row * TL::CH;
            cp_async16(dst + row * TL::UX + 4 * ch, ps.src[k] + zoff);
        }
    }
}

struct PairGeo {
    int lby;           // row in the result region
    int lbx0, lbx1;    // columns of the two points
    int p0, p1;        // result-plane indices lby * BXP + lbx
    int up0, up1;      // staged-plane indices
    int ax0, ax1, ay;  // wrapped global coordinates
    bool isC0, isC1;   // each point is a tile cell inside the box
    bool wx, wy, wz;   // wall rules may apply on this axis (warp-uniform after narrowing)
};

template <class TL>
__device__ __forceinline__ PairGeo pair_geo(const SimParams& P, int x0, int y0, int z0, int z1, int off) {
    PairGeo g;
    const int t = threadIdx.x;
    const bool perx = P.qper[0] && P.qper[1] && P.uper[0] && P.uper[1];
    const bool pery = P.qper[2] && P.qper[3] && P.uper[2] && P.uper[3];
    const bool perz = P.qper[4] && P.qper[5] && P.uper[4] && P.uper[5];
    g.wx = !perx && (x0 - 1 < 1 || x0 + TL::TCX > P.nx - 2);
    g.wy = !pery && (y0 - 1 < 1 || y0 + TL::TCY > P.ny - 2);
    g.wz = !perz && (z0 - 1 < 1 || z1 > P.nz - 2);
    const int j = t % TL::HP, h = t / TL::HP;  // half-row h = 2 warp + half
    const int m = h & 3;
    g.lby = (h & ~3) + (m == 1 ? 2 : m == 2 ? 1 : m);
    g.lbx0 = j;
    g.lbx1 = j + TL::HP;
    g.p0 = g.lby * TL::BXP + g.lbx0;
    g.p1 = g.lby * TL::BXP + g.lbx1;
    g.up0 = (g.lby + 1) * TL::UX + g.lbx0 + off;
    g.up1 = (g.lby + 1) * TL::UX + g.lbx1 + off;
    g.ax0 = wrap_coord(x0 - 1 + g.lbx0, P.nx);
    g.ax1 = wrap_coord(x0 - 1 + g.lbx1, P.nx);
    g.ay = wrap_coord(y0 - 1 + g.lby, P.ny);
    const bool rowC = g.lby >= 1 && g.lby <= TL::TCY && y0 + g.lby - 1 < P.ny;
    g.isC0 = rowC && g.lbx0 >= 1 && g.lbx0 <= TL::TCX && x0 + g.lbx0 - 1 < P.nx;
    g.isC1 = rowC && g.lbx1 >= 1 && g.lbx1 <= TL::TCX && x0 + g.lbx1 - 1 < P.nx;
    return g;
}

// ---- wall rules on each half -------------------------------------------------
struct PairRules {
    AxisRule qx0, qx1, qy;  // both points of a pair share their row
    VRule vx0, vx1, vy;
};

// The halves are taken apart and put back by value (no reference to a half
// chosen at run time), so the pairs stay in registers.
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

// What the point update of plane zb leaves in registers for the force.
struct PairPlane {
    F2 qn[5];   // Q_new
    F2 u[3];    // velocity of the point
    F2 ern[3];  // Ericksen force, negated
    F2 pz[3];   // row stress differenced along z
};

// ---- point update of one plane ------------------------------------------------
// The row stress differenced along x and y goes to the result slot of zb.
template <class TL, bool UPWIND, int RM>
__device__ __forceinline__ void qp_compute_plane(const SimParams& P, const Phys<float>& K, const PairGeo& G,
                                                 const PairRules& R, int z0, int zb, const float* QU, float* Bs,
                                                 PairPlane& out) {
    const bool rx = RM == 1 || (RM == 2 && G.wx), ry = RM == 2 && G.wy, rz = RM == 2 && G.wz;
    constexpr int NQU = TL::NQU, UX = TL::UX, NB = TL::NB;
    const float* Qc = QU + pair_slot<TL>(zb, z0) * 8 * NQU;
    const float* Qm = QU + pair_slot<TL>(zb - 1, z0) * 8 * NQU;
    const float* Qp = QU + pair_slot<TL>(zb + 1, z0) * 8 * NQU;
    const int u0 = G.up0, u1 = G.up1;
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
    for (int comp = 0; comp < 3; ++comp) out.u[comp] = ld2(uc[comp], u0, u1);
    F2 gr[8];
#pragma unroll
    for (int comp = 0; comp < 3; ++comp) {
        const F2 c = out.u[comp];
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
    F2 pxy[6];
    pointwise_q_pair<UPWIND>(K, Q, out.u[0], out.u[1], out.u[2], d, g, out.qn, pxy, out.pz, out.ern);
    float* Bxy = Bs + ((zb - z0) & 1) * 6 * NB;
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        Bxy[k * NB + G.p0] = pxy[k].v.x;
        Bxy[k * NB + G.p1] = pxy[k].v.y;
    }
}

// Body force of the pair's tile cells in plane zc from everything but the +z
// neighbour of the row stress: 2 x (x, y differences - the -z neighbour),
// plus the anchoring corrections, -MU u and the Ericksen force.  cur: plane
// zc at the points; zm_pz: the z-differenced row stress of plane zc - 1.
// zp_clamped: the +z neighbour is the Neumann clamp (plane zc itself, added
// here) rather than plane zc + 1.
template <class TL, int RM>
__device__ __forceinline__ void qp_partial_force(const SimParams& P, const Phys<float>& K, const PairGeo& G,
                                                 const PairRules& R, int x0, int y0, int z0, int zc,
                                                 const float* Bs, const PairPlane& cur, const F2 zm_pz[3],
                                                 F2 part[3], bool& zp_clamped) {
    const bool rx = RM == 1 || (RM == 2 && G.wx), ry = RM == 2 && G.wy, rz = RM == 2 && G.wz;
    constexpr int NB = TL::NB, BXP = TL::BXP;
    const int p0 = G.p0, p1 = G.p1;
    const float* Bxy = Bs + ((zc - z0) & 1) * 6 * NB;
    const int gy = y0 + G.lby - 1;
    AxisRule qz;
    if (rz) qz = q_rule(P, 2, zc, P.nz);
    // Sigma / tau differences with the Neumann/periodic index clamp QXoff
    // (src/offsets.h:59-83, used by PassiveStressDivergence)
    const bool zmc = rz && zc == 0 && !P.qper[4];
    zp_clamped = rz && zc == P.nz - 1 && !P.qper[5];
    F2 f[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float* px = Bxy + a * NB;
        const float* py = Bxy + (3 + a) * NB;
        F2 xm = ld2(px, p0 - 1, p1 - 1), xp = ld2(px, p0 + 1, p1 + 1);
        F2 ym = ld2(py, p0 - BXP, p1 - BXP), yp = ld2(py, p0 + BXP, p1 + BXP);
        if (rx) {
            const int gx0 = x0 + G.lbx0 - 1, gx1 = x0 + G.lbx1 - 1;
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
        const F2 zm = zmc ? cur.pz[a] : zm_pz[a];
        F2 t = ((xp - xm) + (yp - ym)) - zm;
        if (zp_clamped) t = t + cur.pz[a];
        f[a] = t * f2(0.5f);
    }
    // anchoring walls: the Q_new ghost differs from the clamp (anchor_delta)
    const F2* qc = cur.qn;
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
    // Ericksen + f - MU u (ern holds the Ericksen force negated)
    const F2 nMU = f2(-K.MU);
#pragma unroll
    for (int a = 0; a < 3; ++a) part[a] = fma2(nMU, cur.u[a], f[a]) - cur.ern[a];
}

// Marches a block through planes [z0, z1) of the column at (x0, y0).
template <class TL, bool UPWIND, class OutQ, class OutF>
__device__ __forceinline__ void qp_march(const SimParams& P, int x0, int y0, int z0, int z1,
                                         const float* __restrict__ qin, const float* __restrict__ uin, float* smem,
                                         const OutQ& outq, const OutF& outf) {
    float* QU = smem;
    float* Bs = smem + TL::stage_floats;
    const Phys<float>& K = phys_ref<float>(P);
    const int s0 = (x0 - 2) & ~3;  // 16-byte boundary at or below x0 - 2
    const int off = x0 - 1 - s0;   // staged column of result column 0
    PairGeo G = pair_geo<TL>(P, x0, y0, z0, z1, off);
    PairRules R;
    R.qx0 = q_rule(P, 0, G.ax0, P.nx);
    R.qx1 = q_rule(P, 0, G.ax1, P.nx);
    R.vx0 = v_rule(P, 0, G.ax0, P.nx);
    R.vx1 = v_rule(P, 0, G.ax1, P.nx);
    R.qy = q_rule(P, 1, G.ay, P.ny);
    R.vy = v_rule(P, 1, G.ay, P.ny);
    narrow_walls_pair(G, R);
    PairSrc<TL> ps;
    pair_src_init<TL>(P, s0, y0, qin, uin, ps);
    const int rm = (G.wx || G.wy || G.wz) ? ((G.wy || G.wz) ? 2 : 1) : 0;
    // (a macro, not a lambda: a lambda taking the plane structs by reference
    // put them in local memory)
#define LBMAN_QP_COMPUTE(zb, pl)                                                              \
    do {                                                                                      \
        if (rm == 0) qp_compute_plane<TL, UPWIND, 0>(P, K, G, R, z0, zb, QU, Bs, pl);          \
        else if (rm == 1) qp_compute_plane<TL, UPWIND, 1>(P, K, G, R, z0, zb, QU, Bs, pl);     \
        else qp_compute_plane<TL, UPWIND, 2>(P, K, G, R, z0, zb, QU, Bs, pl);                  \
    } while (0)

    // Copy groups: one per plane, in plane order.  Planes z0-2 .. z0+LEAD
    // fill the ring; plane z0+LEAD+1 takes the slot of z0-2 once the update
    // of z0-1 is done; in the loop, iteration zc copies plane zc+LEAD+2 into
    // the slot of plane zc-1 (last read by the update of zc) and waits for
    // plane zc+3, which the next update needs: LEAD-1 newer groups may stay
    // in flight.  Every iteration commits a group (empty near the end of the
    // march) so the counts hold.
    constexpr int LEAD = TL::LEAD;
    for (int z = z0 - 2; z <= z0 + LEAD; ++z) {
        pair_load_plane<TL>(P, z0, z, QU, ps);
        cp_async_commit();
    }
    cp_async_wait_group<LEAD>();  // planes z0-2 .. z0
    __syncthreads();
    PairPlane cur;
    F2 zm_pz[3];
    LBMAN_QP_COMPUTE(z0 - 1, cur);  // only its row stress along z is used
#pragma unroll
    for (int a = 0; a < 3; ++a) zm_pz[a] = cur.pz[a];
    __syncthreads();  // the slot of z0-2 is free again
    if (z0 + LEAD + 1 <= z1 + 1) pair_load_plane<TL>(P, z0, z0 + LEAD + 1, QU, ps);
    cp_async_commit();
    cp_async_wait_group<LEAD>();  // .. z0+1
    __syncthreads();
    LBMAN_QP_COMPUTE(z0, cur);
    cp_async_wait_group<LEAD - 1>();  // .. z0+2
    __syncthreads();
#pragma unroll 1
    for (int zc = z0; zc < z1; ++zc) {
        if (zc + LEAD + 2 <= z1 + 1) pair_load_plane<TL>(P, z0, zc + LEAD + 2, QU, ps);
        cp_async_commit();
        // Force of plane zc without its +z term: reads the x/y row stress of
        // plane zc (complete since the last barrier) and registers.  Only
        // pairs holding a tile cell: their neighbours' result indices lie
        // inside the result planes (a pair of a halo row has none).
        const bool cell = G.isC0 || G.isC1;
        F2 part[3];
        bool zp_clamped = false;
        if (cell) {
            if (rm == 0) qp_partial_force<TL, 0>(P, K, G, R, x0, y0, z0, zc, Bs, cur, zm_pz, part, zp_clamped);
            else if (rm == 1) qp_partial_force<TL, 1>(P, K, G, R, x0, y0, z0, zc, Bs, cur, zm_pz, part, zp_clamped);
            else qp_partial_force<TL, 2>(P, K, G, R, x0, y0, z0, zc, Bs, cur, zm_pz, part, zp_clamped);
        }
        const int64_t row = (int64_t)zc * P.nxy + (int64_t)(y0 + G.lby - 1) * P.nx + x0 - 1;
        if (G.isC0) outq(row + G.lbx0, cur.qn[0].v.x, cur.qn[1].v.x, cur.qn[2].v.x, cur.qn[3].v.x, cur.qn[4].v.x);
        if (G.isC1) outq(row + G.lbx1, cur.qn[0].v.y, cur.qn[1].v.y, cur.qn[2].v.y, cur.qn[3].v.y, cur.qn[4].v.y);
#pragma unroll
        for (int a = 0; a < 3; ++a) zm_pz[a] = cur.pz[a];
        // Update of plane zc + 1 into the other result slot: no barrier
        // needed, nobody reads that slot before the next one.
        LBMAN_QP_COMPUTE(zc + 1, cur);
        if (cell) {
            if (!zp_clamped) {
#pragma unroll
                for (int a = 0; a < 3; ++a) part[a] = fma2(f2(0.5f), cur.pz[a], part[a]);
            }
            if (G.isC0) outf(row + G.lbx0, part[0].v.x, part[1].v.x, part[2].v.x);
            if (G.isC1) outf(row + G.lbx1, part[0].v.y, part[1].v.y, part[2].v.y);
        }
        cp_async_wait_group<LEAD - 1>();  // plane zc+3
        __syncthreads();
    }
#undef LBMAN_QP_COMPUTE
}

// Consumers of the split organisation: Q_new and the body force of one cell.
struct StoreQ2 {
    float* __restrict__ qout;
    int64_t V;
    __device__ __forceinline__ void operator()(int64_t cell, float q0, float q1, float q2, float q3, float q4) const {
        qout[cell] = q0;
        qout[V + cell] = q1;
        qout[2 * V + cell] = q2;
        qout[3 * V + cell] = q3;
        qout[4 * V + cell] = q4;
    }
};
struct StoreF2 {
    float* __restrict__ Fout;
    int64_t V;
    __device__ __forceinline__ void operator()(int64_t cell, float F0, float F1, float F2v) const {
        Fout[cell] = F0;
        Fout[V + cell] = F1;
        Fout[2 * V + cell] = F2v;
    }
};

// The block's work: fixed z chunks or the balanced schedule (qf_run).
template <class TL, bool UPWIND>
__device__ __forceinline__ void qp_run(const SimParams& P, int zc_len, const float* __restrict__ qin,
                                       const float* __restrict__ uin, float* smem, float* __restrict__ qout,
                                       float* __restrict__ Fout) {
    const StoreQ2 oq{qout, P.V};
    const StoreF2 of{Fout, P.V};
    if (zc_len > 0) {
        const int z0 = P.zlo + (int)blockIdx.z * zc_len;
        if (z0 >= P.zhi) return;
        qp_march<TL, UPWIND>(P, blockIdx.x * TL::TCX, blockIdx.y * TL::TCY, z0, min(z0 + zc_len, P.zhi), qin, uin,
                             smem, oq, of);
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
        qp_march<TL, UPWIND>(P, bx * TL::TCX, by * TL::TCY, z0, z1, qin, uin, smem, oq, of);
        __syncthreads();  // the staging rings are reused by the next segment
        w += z1 - z0;
    }
}

template <class TL, bool UPWIND>
__global__ void __launch_bounds__(TL::NT, TL::MINB)
    qpair_kernel(const __grid_constant__ SimParams P, int zc_len, const float* __restrict__ qin,
                 const float* __restrict__ uin, float* __restrict__ qout, float* __restrict__ Fout) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    qp_run<TL, UPWIND>(P, zc_len, qin, uin, reinterpret_cast<float*>(smem_raw), qout, Fout);
}

}  // namespace lbman
