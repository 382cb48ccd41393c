// physics_pair.cuh -- the FP32 Beris-Edwards right-hand side of two points
// at once in packed f32x2 arithmetic (sm_100 FFMA2 / FADD2 / FMUL2), used by
// the two-points-per-thread Q+force kernel (qpair.cuh).
//
// It is pointwise_q_mat of physics.cuh (unhalved first differences, the
// co-rotation and alignment terms as QB + (QB)^T with B = LAMBDA E - W, the
// N = QH products for Sigma and tau), written with explicit fused
// multiply-adds and with Sigma, tau and Q_new combined into the row stress
// the force pass differentiates.  tests/host/pair_check.cpp compiles it as
// host C++ and checks it against the reference-ordered pointwise_q.
#pragma once

#include "common.cuh"

namespace lbman {

// ---- packed pairs ----------------------------------------------------------
struct F2 {
    float2 v;
};
__device__ __forceinline__ F2 f2(float a) { return {make_float2(a, a)}; }
__device__ __forceinline__ F2 f2(float a, float b) { return {make_float2(a, b)}; }
__device__ __forceinline__ F2 operator+(F2 a, F2 b) { return {__fadd2_rn(a.v, b.v)}; }
__device__ __forceinline__ F2 operator*(F2 a, F2 b) { return {__fmul2_rn(a.v, b.v)}; }
// a * b + c
__device__ __forceinline__ F2 fma2(F2 a, F2 b, F2 c) { return {__ffma2_rn(a.v, b.v, c.v)}; }
// a - b in one instruction (b * -1 + a; the product is exact)
__device__ __forceinline__ F2 operator-(F2 a, F2 b) { return {__ffma2_rn(b.v, make_float2(-1.0f, -1.0f), a.v)}; }

struct QD2 {
    F2 dx, dy, dz, lap, d2x, d2y, d2z;
};

// Unhalved first differences, Laplacian, second differences (upwind only).
template <bool UPWIND>
__device__ __forceinline__ QD2 q_derivs2(F2 xm, F2 xp, F2 ym, F2 yp, F2 zm, F2 zp, F2 c) {
    QD2 d;
    d.dx = xp - xm;
    d.dy = yp - ym;
    d.dz = zp - zm;
    const F2 sx = xm + xp, sy = ym + yp, sz = zm + zp;
    d.lap = fma2(f2(-6.0f), c, (sx + sy) + sz);
    if (UPWIND) {
        d.d2x = fma2(f2(-2.0f), c, sx);
        d.d2y = fma2(f2(-2.0f), c, sy);
        d.d2z = fma2(f2(-2.0f), c, sz);
    }
    return d;
}

struct GradU2 {
    F2 ux_x, ux_y, ux_z, uy_x, uy_y, uy_z, uz_x, uz_y;  // unhalved differences
};

// Beris-Edwards right-hand side of two points: Q_new, the row stress
// Pi = Sigma + tau - ALPHA Q_new grouped by differentiation axis (pi_xy[6]:
// the rows differenced along x then y; pi_z[3]: along z), and the Ericksen
// force with the opposite sign (eric_neg = +H : grad Q).
template <bool UPWIND>
__device__ __forceinline__ void pointwise_q_pair(const Phys<float>& K, const F2 Q[5], F2 ux, F2 uy, F2 uz,
                                                 const QD2 d[5], const GradU2& g, F2 qn[5], F2 pi_xy[6],
                                                 F2 pi_z[3], F2 eric_neg[3]) {
    const float LAMBDA = K.LAMBDA, k23 = 2.0f / 3.0f;
    const F2 a = Q[0], b = Q[1], c = Q[2], e = Q[3], h = Q[4];  // Qxx Qxy Qxz Qyy Qyz
    const F2 zz = (a + e) * f2(-1.0f);                          // Qzz

    // advection -u.grad Q with the 1/2 of the unhalved differences folded in
    F2 rhs[5];
    {
        const F2 hx = ux * f2(-0.5f), hy = uy * f2(-0.5f), hz = uz * f2(-0.5f);
        F2 ax, ay, az;
        if (UPWIND) {
            ax = f2(0.5f * fabsf(ux.v.x), 0.5f * fabsf(ux.v.y));
            ay = f2(0.5f * fabsf(uy.v.x), 0.5f * fabsf(uy.v.y));
            az = f2(0.5f * fabsf(uz.v.x), 0.5f * fabsf(uz.v.y));
        }
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            F2 t = fma2(hz, d[k].dz, fma2(hy, d[k].dy, hx * d[k].dx));
            if (UPWIND) t = fma2(az, d[k].d2z, fma2(ay, d[k].d2y, fma2(ax, d[k].d2x, t)));
            rhs[k] = t;
        }
    }
    // co-rotation + alignment = QB + (QB)^T - 2 tr(QB) Q + LAMBDA (2/3) E,
    // B = LAMBDA E - W; E, W from the unhalved gradients (factors 1/2, 1/4)
    {
        const F2 lm = f2(0.25f * (LAMBDA - 1.0f)), lp = f2(0.25f * (LAMBDA + 1.0f));
        const F2 Bxx = f2(0.5f * LAMBDA) * g.ux_x, Byy = f2(0.5f * LAMBDA) * g.uy_y;
        const F2 Bzz = (Bxx + Byy) * f2(-1.0f);
        const F2 Bxy = fma2(lm, g.ux_y, lp * g.uy_x), Byx = fma2(lp, g.ux_y, lm * g.uy_x);
        const F2 Bxz = fma2(lm, g.ux_z, lp * g.uz_x), Bzx = fma2(lp, g.ux_z, lm * g.uz_x);
        const F2 Byz = fma2(lm, g.uy_z, lp * g.uz_y), Bzy = fma2(lp, g.uy_z, lm * g.uz_y);
        // N = Q B
        const F2 Nxx = fma2(c, Bzx, fma2(b, Byx, a * Bxx));
        const F2 Nyy = fma2(h, Bzy, fma2(e, Byy, b * Bxy));
        const F2 Nzz = fma2(zz, Bzz, fma2(h, Byz, c * Bxz));
        const F2 T = (Nxx + Nyy) + Nzz;  // LAMBDA tr(QE)
        const F2 m2 = T * f2(-2.0f), nkT = T * f2(-k23);
        const float lk = LAMBDA * k23;
        rhs[0] = rhs[0] + fma2(m2, a, fma2(f2(0.5f * lk), g.ux_x, fma2(f2(2.0f), Nxx, nkT)));
        rhs[3] = rhs[3] + fma2(m2, e, fma2(f2(0.5f * lk), g.uy_y, fma2(f2(2.0f), Nyy, nkT)));
        const F2 lk4 = f2(0.25f * lk);
        const F2 Nxy = fma2(c, Bzy, fma2(b, Byy, a * Bxy)), Nyx = fma2(h, Bzx, fma2(e, Byx, b * Bxx));
        rhs[1] = rhs[1] + fma2(m2, b, fma2(lk4, g.ux_y + g.uy_x, Nxy + Nyx));
        const F2 Nxz = fma2(c, Bzz, fma2(b, Byz, a * Bxz)), Nzx = fma2(zz, Bzx, fma2(h, Byx, c * Bxx));
        rhs[2] = rhs[2] + fma2(m2, c, fma2(lk4, g.ux_z + g.uz_x, Nxz + Nzx));
        const F2 Nyz = fma2(h, Bzz, fma2(e, Byz, b * Bxz)), Nzy = fma2(zz, Bzy, fma2(h, Byy, c * Bxy));
        rhs[4] = rhs[4] + fma2(m2, h, fma2(lk4, g.uy_z + g.uz_y, Nyz + Nzy));
    }
    // molecular field H = L lap Q - (A + C tr Q^2) Q - B [Q^2]_traceless
    F2 H[5];
    {
        const F2 s = fma2(h, h, fma2(c, c, fma2(b, b, fma2(a, e, fma2(e, e, a * a)))));  // tr(Q^2) / 2
        const F2 t3 = s * f2(2.0f / 3.0f);                                              // tr(Q^2) / 3
        const F2 nld = fma2(f2(-2.0f * K.C), s, f2(-K.A));                              // -(A + C tr Q^2)
        const F2 L = f2(K.L), nB = f2(-K.B), B = f2(K.B);
        const F2 X0 = fma2(c, c, fma2(b, b, a * a)) - t3;
        const F2 X3 = fma2(h, h, fma2(e, e, b * b)) - t3;
        const F2 X1 = fma2(c, h, fma2(b, e, a * b));
        H[0] = fma2(L, d[0].lap, fma2(nld, a, nB * X0));
        H[1] = fma2(L, d[1].lap, fma2(nld, b, nB * X1));
        // -B (b h - c e) = (-B b) h + (B c) e
        H[2] = fma2(L, d[2].lap, fma2(nld, c, fma2(nB * b, h, (B * c) * e)));
        H[3] = fma2(L, d[3].lap, fma2(nld, e, nB * X3));
        // -B (b c - h a) = (-B b) c + (B h) a
        H[4] = fma2(L, d[4].lap, fma2(nld, h, fma2(nB * b, c, (B * h) * a)));
    }
    const F2 Hxx = H[0], Hxy = H[1], Hxz = H[2], Hyy = H[3], Hyz = H[4];
    const F2 Hzz = (Hxx + Hyy) * f2(-1.0f);

    // H : grad Q with the doubled differences:
    // sum_k H_k d_k + (Hxx d3 + Hyy d0) / 2 = Hxx (d0 + d3/2) + Hyy (d3 + d0/2) + ...
    {
        const F2 hf = f2(0.5f);
        eric_neg[0] = fma2(Hyz, d[4].dx, fma2(Hxz, d[2].dx, fma2(Hxy, d[1].dx,
                      fma2(Hyy, fma2(hf, d[0].dx, d[3].dx), Hxx * fma2(hf, d[3].dx, d[0].dx)))));
        eric_neg[1] = fma2(Hyz, d[4].dy, fma2(Hxz, d[2].dy, fma2(Hxy, d[1].dy,
                      fma2(Hyy, fma2(hf, d[0].dy, d[3].dy), Hxx * fma2(hf, d[3].dy, d[0].dy)))));
        eric_neg[2] = fma2(Hyz, d[4].dz, fma2(Hxz, d[2].dz, fma2(Hxy, d[1].dz,
                      fma2(Hyy, fma2(hf, d[0].dz, d[3].dz), Hxx * fma2(hf, d[3].dz, d[0].dz)))));
    }
    {
        const F2 G = f2(K.GAMMA), DT = f2(K.DT);
#pragma unroll
        for (int k = 0; k < 5; ++k) qn[k] = fma2(DT, fma2(G, H[k], rhs[k]), Q[k]);
    }
    // N = Q H; Sigma = -2/3 LAMBDA H - LAMBDA (N + N^T) + LAMBDA tr(N) (2/3 I + 2 Q)
    // (diagonal), tau = N - N^T; then the row stress Pi = Sigma + tau - ALPHA Q_new
    {
        const F2 mk23L = f2(-k23 * LAMBDA), mL = f2(-LAMBDA), m2L = f2(-2.0f * LAMBDA);
        const F2 nA = f2(-K.ALPHA);
        const F2 Nxx = fma2(c, Hxz, fma2(b, Hxy, a * Hxx));
        const F2 Nyy = fma2(h, Hyz, fma2(e, Hyy, b * Hxy));
        const F2 Nzz = fma2(zz, Hzz, fma2(h, Hyz, c * Hxz));
        const F2 lt = ((Nxx + Nyy) + Nzz) * f2(LAMBDA);
        const F2 lt2 = lt + lt;
        const F2 s0 = fma2(mk23L, Hxx, fma2(m2L, Nxx, lt * fma2(f2(2.0f), a, f2(k23))));
        const F2 s3 = fma2(mk23L, Hyy, fma2(m2L, Nyy, lt * fma2(f2(2.0f), e, f2(k23))));
        const F2 Nxy = fma2(c, Hyz, fma2(b, Hyy, a * Hxy)), Nyx = fma2(h, Hxz, fma2(e, Hxy, b * Hxx));
        const F2 t0 = Nxy - Nyx;
        const F2 s1 = fma2(mk23L, Hxy, fma2(mL, Nxy + Nyx, lt2 * b));
        const F2 Nxz = fma2(c, Hzz, fma2(b, Hyz, a * Hxz)), Nzx = fma2(zz, Hxz, fma2(h, Hxy, c * Hxx));
        const F2 t1 = Nxz - Nzx;
        const F2 s2 = fma2(mk23L, Hxz, fma2(mL, Nxz + Nzx, lt2 * c));
        const F2 Nyz = fma2(h, Hzz, fma2(e, Hyz, b * Hxz)), Nzy = fma2(zz, Hyz, fma2(h, Hyy, c * Hxy));
        const F2 t2 = Nyz - Nzy;
        const F2 s4 = fma2(mk23L, Hyz, fma2(mL, Nyz + Nzy, lt2 * h));
        pi_xy[0] = fma2(nA, qn[0], s0);
        pi_xy[1] = fma2(nA, qn[1], s1 - t0);
        pi_xy[2] = fma2(nA, qn[2], s2 - t1);
        pi_xy[3] = fma2(nA, qn[1], s1 + t0);
        pi_xy[4] = fma2(nA, qn[3], s3);
        pi_xy[5] = fma2(nA, qn[4], s4 - t2);
        pi_z[0] = fma2(nA, qn[2], s2 + t1);
        pi_z[1] = fma2(nA, qn[4], s4 + t2);
        pi_z[2] = fma2(nA, qn[0] + qn[3], s0 + s3) * f2(-1.0f);
    }
}

}  // namespace lbman
