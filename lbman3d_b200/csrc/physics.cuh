// physics.cuh -- pointwise Beris-Edwards / D3Q15 physics and the wall ghost
// rules, templated on the compute type R.
//
// The FP64 instantiation is compiled with --fmad=false and keeps the
// association order of the reference's expressions term for term
// (src/model.h:102-361, src/physics_helpers.h:69-129,
// src/boundary_handler.h:112-392), so its results are bitwise equal to the
// reference CPU solver.  The FP32 instantiation is the same algebra with
// contraction allowed.  Halving is written as a multiplication by 0.5, which
// is exact and therefore identical to the reference's division by 2.0.
#pragma once

#include "common.cuh"

namespace lbman {

// First/second differences of one Q component (QDerivs, src/qtensor_types.h:304).
template <class R>
struct QD {
    R dx, dy, dz, lap, d2x, d2y, d2z;
};

// Wall handling of one axis at one point, decided once per point and reused
// for every component: SafeFetchAxisOffset + QAxisGhostPair for Q
// (src/boundary_handler.h:76-89, 253-282), VelocityAxisGhostPair for u
// (src/boundary_handler.h:135-146).
struct AxisRule {
    bool m_clamp, p_clamp;    // take the centre value instead of the image
    bool m_ghost, p_ghost;    // then replace by the face's ghost rule
    int lo, hi;               // face indices
};

__device__ __forceinline__ AxisRule q_rule(const SimParams& P, int ax, int a, int n) {
    AxisRule r;
    r.lo = 2 * ax;
    r.hi = r.lo + 1;
    r.m_clamp = a == 0 && !P.qper[r.lo];
    r.p_clamp = a == n - 1 && !P.qper[r.hi];
    // the Lo tag decides whether ghosts apply on this axis
    r.m_ghost = !P.qper[r.lo] && a == 0 && P.face[r.lo].qbc == Q_ANCHORING;
    r.p_ghost = !P.qper[r.lo] && a == n - 1 && P.face[r.hi].qbc == Q_ANCHORING;
    // a Neumann (or Periodic-tagged) ghost equals the centre, i.e. a clamp
    if (!P.qper[r.lo]) {
        if (a == 0) r.m_clamp = true;
        if (a == n - 1) r.p_clamp = true;
    }
    return r;
}

template <class R>
__device__ __forceinline__ void q_apply(const AxisRule& r, const Phys<R>& K, int comp, R c, R& m, R& p) {
    if (r.m_clamp) m = c;
    if (r.p_clamp) p = c;
    if (r.m_ghost) m = R(2.0) * K.anchor[r.lo][comp] - c;
    if (r.p_ghost) p = R(2.0) * K.anchor[r.hi][comp] - c;
}

struct VRule {
    bool m_clamp, p_clamp, m_wall, p_wall;
    int lo, hi;
};

__device__ __forceinline__ VRule v_rule(const SimParams& P, int ax, int a, int n) {
    VRule r;
    r.lo = 2 * ax;
    r.hi = r.lo + 1;
    r.m_clamp = a == 0 && !P.uper[r.lo];
    r.p_clamp = a == n - 1 && !P.uper[r.hi];
    r.m_wall = !P.uper[r.lo] && a == 0;
    r.p_wall = !P.uper[r.lo] && a == n - 1;
    return r;
}

// VelocityGhost (src/boundary_handler.h:121-130).
template <class R>
__device__ __forceinline__ R v_ghost(const SimParams& P, const Phys<R>& K, int face, int comp, R vb,
                                     bool normal) {
    const int ubc = P.face[face].ubc;
    const R wall = ubc == U_MOVING ? K.uw[face][comp] : R(0.0);
    if (ubc == U_SPECULAR) return normal ? (R(2.0) * wall - vb) : vb;
    return R(2.0) * wall - vb;
}

// VelocityAxisGradient (src/boundary_handler.h:157-163); HALF = false
// returns the unhalved difference.
template <class R, bool HALF = true>
__device__ __forceinline__ R v_grad(const SimParams& P, const Phys<R>& K, const VRule& r, int comp, R m,
                                    R c, R p, bool normal) {
    if (r.m_clamp) m = c;
    if (r.p_clamp) p = c;
    if (r.m_wall) m = v_ghost<R>(P, K, r.lo, comp, c, normal);
    if (r.p_wall) p = v_ghost<R>(P, K, r.hi, comp, c, normal);
    return HALF ? R(0.5) * (p - m) : (p - m);
}

// HALF = false keeps the first differences unhalved (2x the centred
// difference), for the FP32 right-hand side that folds the 1/2 into its
// coefficients.
template <class R, bool HALF = true>
__device__ __forceinline__ QD<R> q_derivs(R xm, R xp, R ym, R yp, R zm, R zp, R c) {
    QD<R> d;
    d.dx = HALF ? R(0.5) * (xp - xm) : (xp - xm);
    d.dy = HALF ? R(0.5) * (yp - ym) : (yp - ym);
    d.dz = HALF ? R(0.5) * (zp - zm) : (zp - zm);
    d.lap = (xm + xp + ym + yp + zm + zp) - R(6.0) * c;
    d.d2x = (xm + xp) - R(2.0) * c;
    d.d2y = (ym + yp) - R(2.0) * c;
    d.d2z = (zm + zp) - R(2.0) * c;
    return d;
}

template <class R>
struct GradU {
    R ux_x, ux_y, ux_z, uy_x, uy_y, uy_z, uz_x, uz_y;
};

// AdvectiveAxisTerm / AdvectiveDerivative (src/model.h:60-82).
template <class R, bool UPWIND>
__device__ __forceinline__ R adv_axis(R u, R dq, R d2q) {
    if (UPWIND) {
        const R au = u < R(0.0) ? -u : u;
        return u * dq - R(0.5) * au * d2q;
    }
    return u * dq;
}
template <class R, bool UPWIND>
__device__ __forceinline__ R adv_deriv(R ux, R uy, R uz, const QD<R>& d) {
    return adv_axis<R, UPWIND>(ux, d.dx, d.d2x) + adv_axis<R, UPWIND>(uy, d.dy, d.d2y) +
           adv_axis<R, UPWIND>(uz, d.dz, d.d2z);
}

// PointwiseStepAndSetupBodyForce (src/model.h:102-342): Q_new, Sigma, tau and
// the Ericksen force -H:grad Q at one cell.
template <class R, bool UPWIND>
__device__ __forceinline__ void pointwise_q(const Phys<R>& K, const R Q[5], R ux, R uy, R uz,
                                            const QD<R> d[5], const GradU<R>& g, R qn[5], R sig[5],
                                            R tau[3], R eric[3]) {
    const R A = K.A, B = K.B, C = K.C, L = K.L, LAMBDA = K.LAMBDA, GAMMA = K.GAMMA, DT = K.DT;
    const R Qxx = Q[0], Qxy = Q[1], Qxz = Q[2], Qyy = Q[3], Qyz = Q[4];

    const R TrQ2 = R(2.0) * (Qxx * Qxx + Qyy * Qyy + Qxx * Qyy + Qxy * Qxy + Qxz * Qxz + Qyz * Qyz);
    const R k13 = R(1.0 / 3.0);
    const R Q2_xx = Qxx * Qxx + Qxy * Qxy + Qxz * Qxz - k13 * TrQ2;
    const R Q2_xy = Qxx * Qxy + Qxy * Qyy + Qxz * Qyz;
    const R Q2_xz = Qxy * Qyz - Qxz * Qyy;
    const R Q2_yy = Qxy * Qxy + Qyy * Qyy + Qyz * Qyz - k13 * TrQ2;
    const R Q2_yz = Qxy * Qxz - Qyz * Qxx;

    const R Exx = g.ux_x;
    const R Exy = R(0.5) * (g.ux_y + g.uy_x);
    const R Exz = R(0.5) * (g.ux_z + g.uz_x);
    const R Eyy = g.uy_y;
    const R Eyz = R(0.5) * (g.uy_z + g.uz_y);
    const R Wxy = R(0.5) * (g.ux_y - g.uy_x);
    const R Wxz = R(0.5) * (g.ux_z - g.uz_x);
    const R Wyz = R(0.5) * (g.uy_z - g.uz_y);

    const R adv_xx = -adv_deriv<R, UPWIND>(ux, uy, uz, d[0]);
    const R adv_xy = -adv_deriv<R, UPWIND>(ux, uy, uz, d[1]);
    const R adv_xz = -adv_deriv<R, UPWIND>(ux, uy, uz, d[2]);
    const R adv_yy = -adv_deriv<R, UPWIND>(ux, uy, uz, d[3]);
    const R adv_yz = -adv_deriv<R, UPWIND>(ux, uy, uz, d[4]);

    const R cor_xx = R(2.0) * (Qxy * Wxy + Qxz * Wxz);
    const R cor_xy = -Qxx * Wxy + Qxz * Wyz + Qyy * Wxy + Qyz * Wxz;
    const R cor_xz = R(-2.0) * Qxx * Wxz - Qxy * Wyz - Qyy * Wxz + Qyz * Wxy;
    const R cor_yy = R(2.0) * (-Qxy * Wxy + Qyz * Wyz);
    const R cor_yz = -Qxx * Wyz - Qxy * Wxz - Qxz * Wxy - R(2.0) * Qyy * Wyz;

    const R k23 = R(2.0 / 3.0);
    const R tr_QE = (R(2.0) * Exx + Eyy) * Qxx + (R(2.0) * Exy) * Qxy + (R(2.0) * Exz) * Qxz +
                    (Exx + R(2.0) * Eyy) * Qyy + R(2.0) * Eyz * Qyz;
    const R aln2_xx = R(2.0) * (Exx * Qxx + Exy * Qxy + Exz * Qxz) - k23 * tr_QE;
    const R aln2_xy = Exy * Qxx + Eyy * Qxy + Eyz * Qxz + Qxy * Exx + Qyy * Exy + Qyz * Exz;
    const R aln2_xz =
        Exz * Qxx + Eyz * Qxy + (-Exx - Eyy) * Qxz + Qxz * Exx + Qyz * Exy + (-Qxx - Qyy) * Exz;
    const R aln2_yy = R(2.0) * (Exy * Qxy + Eyy * Qyy + Eyz * Qyz) - k23 * tr_QE;
    const R aln2_yz =
        Exz * Qxy + Eyz * Qyy + (-Exx - Eyy) * Qyz + Qxz * Exy + Qyz * Eyy + (-Qxx - Qyy) * Eyz;
    const R aln3_xx = R(-2.0) * tr_QE * Qxx;
    const R aln3_xy = R(-2.0) * tr_QE * Qxy;
    const R aln3_xz = R(-2.0) * tr_QE * Qxz;
    const R aln3_yy = R(-2.0) * tr_QE * Qyy;
    const R aln3_yz = R(-2.0) * tr_QE * Qyz;

    const R ld = A + C * TrQ2;
    const R Hxx = L * d[0].lap - ld * Qxx - B * Q2_xx;
    const R Hxy = L * d[1].lap - ld * Qxy - B * Q2_xy;
    const R Hxz = L * d[2].lap - ld * Qxz - B * Q2_xz;
    const R Hyy = L * d[3].lap - ld * Qyy - B * Q2_yy;
    const R Hyz = L * d[4].lap - ld * Qyz - B * Q2_yz;

    eric[0] = R(-2.0) * (Hxx * d[0].dx + Hxy * d[1].dx + Hxz * d[2].dx + Hyy * d[3].dx + Hyz * d[4].dx) -
              Hxx * d[3].dx - Hyy * d[0].dx;
    eric[1] = R(-2.0) * (Hxx * d[0].dy + Hxy * d[1].dy + Hxz * d[2].dy + Hyy * d[3].dy + Hyz * d[4].dy) -
              Hxx * d[3].dy - Hyy * d[0].dy;
    eric[2] = R(-2.0) * (Hxx * d[0].dz + Hxy * d[1].dz + Hxz * d[2].dz + Hyy * d[3].dz + Hyz * d[4].dz) -
              Hxx * d[3].dz - Hyy * d[0].dz;

    const R tr_QH = (R(2.0) * Hxx + Hyy) * Qxx + (R(2.0) * Hxy) * Qxy + (R(2.0) * Hxz) * Qxz +
                    (Hxx + R(2.0) * Hyy) * Qyy + R(2.0) * Hyz * Qyz;
    const R QHxx = R(2.0) * (Hxx * Qxx + Hxy * Qxy + Hxz * Qxz) - k23 * tr_QH;
    const R QHxy = Hxy * Qxx + Hyy * Qxy + Hyz * Qxz + Qxy * Hxx + Qyy * Hxy + Qyz * Hxz;
    const R QHxz =
        Hxz * Qxx + Hyz * Qxy + (-Hxx - Hyy) * Qxz + Qxz * Hxx + Qyz * Hxy + (-Qxx - Qyy) * Hxz;
    const R QHyy = R(2.0) * (Hxy * Qxy + Hyy * Qyy + Hyz * Qyz) - k23 * tr_QH;
    const R QHyz =
        Hxz * Qxy + Hyz * Qyy + (-Hxx - Hyy) * Qyz + Qxz * Hxy + Qyz * Hyy + (-Qxx - Qyy) * Hyz;

    tau[0] = (Hxy * Qxx + Hyy * Qxy + Hyz * Qxz) - (Qxy * Hxx + Qyy * Hxy + Qyz * Hxz);
    tau[1] = (Hxz * Qxx + Hyz * Qxy + (-Hxx - Hyy) * Qxz) - (Qxz * Hxx + Qyz * Hxy + (-Qxx - Qyy) * Hxz);
    tau[2] = (Hxz * Qxy + Hyz * Qyy + (-Hxx - Hyy) * Qyz) - (Qxz * Hxy + Qyz * Hyy + (-Qxx - Qyy) * Hyz);

    const R mk23L = -k23 * LAMBDA;
    const R twoL = R(2.0) * LAMBDA;
    sig[0] = mk23L * Hxx - LAMBDA * QHxx + twoL * tr_QH * Qxx;
    sig[1] = mk23L * Hxy - LAMBDA * QHxy + twoL * tr_QH * Qxy;
    sig[2] = mk23L * Hxz - LAMBDA * QHxz + twoL * tr_QH * Qxz;
    sig[3] = mk23L * Hyy - LAMBDA * QHyy + twoL * tr_QH * Qyy;
    sig[4] = mk23L * Hyz - LAMBDA * QHyz + twoL * tr_QH * Qyz;

    qn[0] = Qxx + DT * (adv_xx + cor_xx + LAMBDA * (k23 * Exx + aln2_xx + aln3_xx) + GAMMA * Hxx);
    qn[1] = Qxy + DT * (adv_xy + cor_xy + LAMBDA * (k23 * Exy + aln2_xy + aln3_xy) + GAMMA * Hxy);
    qn[2] = Qxz + DT * (adv_xz + cor_xz + LAMBDA * (k23 * Exz + aln2_xz + aln3_xz) + GAMMA * Hxz);
    qn[3] = Qyy + DT * (adv_yy + cor_yy + LAMBDA * (k23 * Eyy + aln2_yy + aln3_yy) + GAMMA * Hyy);
    qn[4] = Qyz + DT * (adv_yz + cor_yz + LAMBDA * (k23 * Eyz + aln2_yz + aln3_yz) + GAMMA * Hyz);
}

// The same right-hand side for the FP32 instantiations, with less arithmetic
// (the values agree with the reference's term-by-term expansion, which the
// FP64 path keeps for bitwise parity, to rounding):
//  * d[k].dx/dy/dz and g are the UNHALVED first differences (2x the centred
//    differences); the 1/2 is folded into the coefficients that use them;
//  * co-rotation and alignment together, (WQ - QW) + LAMBDA (QE + EQ), are
//    QB + (QB)^T with B = LAMBDA E - W (Q symmetric, W antisymmetric), and
//    tr(QB) = LAMBDA tr(QE);
//  * for N = QH, QH + HQ = N + N^T and tau = QH - HQ = N - N^T.
template <class R, bool UPWIND>
__device__ __forceinline__ void pointwise_q_mat(const Phys<R>& K, const R Q[5], R ux, R uy, R uz,
                                                const QD<R> d[5], const GradU<R>& g, R qn[5], R sig[5],
                                                R tau[3], R eric[3]) {
    const R A = K.A, B = K.B, C = K.C, L = K.L, LAMBDA = K.LAMBDA, GAMMA = K.GAMMA, DT = K.DT;
    const R a = Q[0], b = Q[1], c = Q[2], e = Q[3], h = Q[4];  // Qxx Qxy Qxz Qyy Qyz
    const R zz = -(a + e);                                     // Qzz
    const R k23 = R(2.0 / 3.0);

    // rhs_k: advection + co-rotation + LAMBDA (alignment), per component.
    R rhs[5];
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        R t = ux * d[k].dx + uy * d[k].dy + uz * d[k].dz;
        if (UPWIND) {
            const R ax = ux < R(0.0) ? -ux : ux, ay = uy < R(0.0) ? -uy : uy, az = uz < R(0.0) ? -uz : uz;
            t = t - (ax * d[k].d2x + ay * d[k].d2y + az * d[k].d2z);
        }
        rhs[k] = R(-0.5) * t;
    }
    {
        const R Exx = R(0.5) * g.ux_x, Eyy = R(0.5) * g.uy_y;
        const R Exy = R(0.25) * (g.ux_y + g.uy_x);
        const R Exz = R(0.25) * (g.ux_z + g.uz_x);
        const R Eyz = R(0.25) * (g.uy_z + g.uz_y);
        const R Wxy = R(0.25) * (g.ux_y - g.uy_x);
        const R Wxz = R(0.25) * (g.ux_z - g.uz_x);
        const R Wyz = R(0.25) * (g.uy_z - g.uz_y);
        const R Bxx = LAMBDA * Exx, Byy = LAMBDA * Eyy, Bzz = -(Bxx + Byy);
        const R Bxy = LAMBDA * Exy - Wxy, Byx = LAMBDA * Exy + Wxy;
        const R Bxz = LAMBDA * Exz - Wxz, Bzx = LAMBDA * Exz + Wxz;
        const R Byz = LAMBDA * Eyz - Wyz, Bzy = LAMBDA * Eyz + Wyz;
        // N = Q B
        const R Nxx = a * Bxx + b * Byx + c * Bzx, Nyy = b * Bxy + e * Byy + h * Bzy;
        const R Nzz = c * Bxz + h * Byz + zz * Bzz;
        const R T = Nxx + Nyy + Nzz;  // LAMBDA tr(QE)
        const R kT = k23 * T, m2 = R(-2.0) * T;
        const R lk = LAMBDA * k23;
        rhs[0] += (R(2.0) * Nxx - kT) + lk * Exx + m2 * a;
        rhs[3] += (R(2.0) * Nyy - kT) + lk * Eyy + m2 * e;
        const R Nxy = a * Bxy + b * Byy + c * Bzy, Nyx = b * Bxx + e * Byx + h * Bzx;
        rhs[1] += (Nxy + Nyx) + lk * Exy + m2 * b;
        const R Nxz = a * Bxz + b * Byz + c * Bzz, Nzx = c * Bxx + h * Byx + zz * Bzx;
        rhs[2] += (Nxz + Nzx) + lk * Exz + m2 * c;
        const R Nyz = b * Bxz + e * Byz + h * Bzz, Nzy = c * Bxy + h * Byy + zz * Bzy;
        rhs[4] += (Nyz + Nzy) + lk * Eyz + m2 * h;
    }

    R H[5];
    {
        const R TrQ2 = R(2.0) * (a * a + e * e + a * e + b * b + c * c + h * h);
        const R t3 = R(1.0 / 3.0) * TrQ2;
        const R ld = A + C * TrQ2;
        H[0] = L * d[0].lap - ld * a - B * (a * a + b * b + c * c - t3);
        H[1] = L * d[1].lap - ld * b - B * (a * b + b * e + c * h);
        H[2] = L * d[2].lap - ld * c - B * (b * h - c * e);
        H[3] = L * d[3].lap - ld * e - B * (b * b + e * e + h * h - t3);
        H[4] = L * d[4].lap - ld * h - B * (b * c - h * a);
    }
    const R Hxx = H[0], Hxy = H[1], Hxz = H[2], Hyy = H[3], Hyz = H[4], Hzz = -(Hxx + Hyy);

    // -H : grad Q with the doubled differences: -2 sum_k H_k d_k - (Hxx d3 + Hyy d0)
    eric[0] = -(Hxx * d[0].dx + Hxy * d[1].dx + Hxz * d[2].dx + Hyy * d[3].dx + Hyz * d[4].dx) -
              R(0.5) * (Hxx * d[3].dx + Hyy * d[0].dx);
    eric[1] = -(Hxx * d[0].dy + Hxy * d[1].dy + Hxz * d[2].dy + Hyy * d[3].dy + Hyz * d[4].dy) -
              R(0.5) * (Hxx * d[3].dy + Hyy * d[0].dy);
    eric[2] = -(Hxx * d[0].dz + Hxy * d[1].dz + Hxz * d[2].dz + Hyy * d[3].dz + Hyz * d[4].dz) -
              R(0.5) * (Hxx * d[3].dz + Hyy * d[0].dz);

#pragma unroll
    for (int k = 0; k < 5; ++k) qn[k] = Q[k] + DT * (rhs[k] + GAMMA * H[k]);

    // N = Q H; sig = -2/3 LAMBDA H - LAMBDA (QH + HQ - 2/3 tr(QH) I) + 2 LAMBDA tr(QH) Q
    const R Nxx = a * Hxx + b * Hxy + c * Hxz, Nyy = b * Hxy + e * Hyy + h * Hyz;
    const R Nzz = c * Hxz + h * Hyz + zz * Hzz;
    const R lt = LAMBDA * (Nxx + Nyy + Nzz);
    const R mk23L = -k23 * LAMBDA;
    sig[0] = mk23L * Hxx - LAMBDA * (R(2.0) * Nxx) + lt * (k23 + R(2.0) * a);
    sig[3] = mk23L * Hyy - LAMBDA * (R(2.0) * Nyy) + lt * (k23 + R(2.0) * e);
    const R Nxy = a * Hxy + b * Hyy + c * Hyz, Nyx = b * Hxx + e * Hxy + h * Hxz;
    tau[0] = Nxy - Nyx;
    sig[1] = mk23L * Hxy - LAMBDA * (Nxy + Nyx) + R(2.0) * lt * b;
    const R Nxz = a * Hxz + b * Hyz + c * Hzz, Nzx = c * Hxx + h * Hxy + zz * Hxz;
    tau[1] = Nxz - Nzx;
    sig[2] = mk23L * Hxz - LAMBDA * (Nxz + Nzx) + R(2.0) * lt * c;
    const R Nyz = b * Hxz + e * Hyz + h * Hzz, Nzy = c * Hxy + h * Hyy + zz * Hyz;
    tau[2] = Nyz - Nzy;
    sig[4] = mk23L * Hyz - LAMBDA * (Nyz + Nzy) + R(2.0) * lt * h;
}

// PointwiseSetActiveStressAndComputeBodyForce + PassiveStressDivergence sums
// (src/model.h:344-361, src/boundary_handler.h:379-391): the force added to
// the Ericksen seed.  dS[axis][comp] are the centred differences of the 5
// Sigma components, dT[axis][comp] of the 3 tau components.
template <class R>
__device__ __forceinline__ void active_passive_force(const Phys<R>& K, const R dQ[5][3], const R dS[3][5],
                                                     const R dT[3][3], R ux, R uy, R uz, const R eric[3],
                                                     R F[3]) {
    const R ALPHA = K.ALPHA, MU = K.MU;
    // f_x = d_x S_xx + d_y(S_xy + T_xy) + d_z(S_xz + T_xz), ... (row convention)
    const R dz_Szz = -(dS[2][0] + dS[2][3]);
    const R pdx = dS[0][0] + (dS[1][1] + dT[1][0]) + (dS[2][2] + dT[2][1]);
    const R pdy = (dS[0][1] - dT[0][0]) + dS[1][3] + (dS[2][4] + dT[2][2]);
    const R pdz = (dS[0][2] - dT[0][1]) + (dS[1][4] - dT[1][2]) + dz_Szz;
    const R fx = -ALPHA * (dQ[0][0] + dQ[1][1] + dQ[2][2]) + pdx - MU * ux;
    const R fy = -ALPHA * (dQ[1][0] + dQ[3][1] + dQ[4][2]) + pdy - MU * uy;
    const R fz = -ALPHA * (dQ[2][0] + dQ[4][1] - dQ[0][2] - dQ[3][2]) + pdz - MU * uz;
    F[0] = eric[0] + fx;
    F[1] = eric[1] + fy;
    F[2] = eric[2] + fz;
}

}  // namespace lbman
