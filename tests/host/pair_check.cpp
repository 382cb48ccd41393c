// Compiles the packed two-point right-hand side (physics_pair.cuh
// pointwise_q_pair, FP32) as host C++ and checks it against the
// reference-ordered one (pointwise_q of physics.cuh) evaluated in double for
// each of the two points separately, on random states, centred and upwind:
// Q_new, the row stress Pi = Sigma + tau - ALPHA Q_new per differentiation
// axis and the Ericksen force (returned negated).  FP32 rounding only: exit 0
// iff every output agrees to 2e-5 of the largest output.
#define __device__
#define __host__
#define __forceinline__ inline
#define __global__
#include <cmath>
#include <cstdio>
#include <random>
#include "common.cuh"
#include "physics.cuh"
#include "physics_pair.cuh"
using namespace lbman;

// The 17 outputs of one point from the reference-ordered form, in the order
// of the packed function: qn[5], Pi_xy[6], Pi_z[3], -eric[3].
template <bool UP>
void reference(const Phys<double>& K, const double Q[5], double ux, double uy, double uz, const QD<double> d[5],
               const GradU<double>& g, double out[17]) {
    double qn[5], sg[5], ta[3], er[3];
    pointwise_q<double, UP>(K, Q, ux, uy, uz, d, g, qn, sg, ta, er);
    const double a = -K.ALPHA;
    for (int k = 0; k < 5; ++k) out[k] = qn[k];
    out[5] = sg[0] + a * qn[0];
    out[6] = (sg[1] - ta[0]) + a * qn[1];
    out[7] = (sg[2] - ta[1]) + a * qn[2];
    out[8] = (sg[1] + ta[0]) + a * qn[1];
    out[9] = sg[3] + a * qn[3];
    out[10] = (sg[4] - ta[2]) + a * qn[4];
    out[11] = (sg[2] + ta[1]) + a * qn[2];
    out[12] = (sg[4] + ta[2]) + a * qn[4];
    out[13] = -(sg[0] + sg[3]) - a * (qn[0] + qn[3]);
    for (int k = 0; k < 3; ++k) out[14 + k] = -er[k];
}

int main() {
    std::mt19937_64 rng(7);
    std::uniform_real_distribution<double> U(-1, 1);
    double worst = 0, scale = 0;
    for (int trial = 0; trial < 4000; ++trial) {
        const bool up = trial & 1;
        Phys<double> K{};
        K.A = 0.5 * (U(rng) + 1); K.B = U(rng); K.C = 0.5 * (U(rng) + 1); K.L = 0.1 * (U(rng) + 1);
        K.LAMBDA = U(rng); K.GAMMA = U(rng) + 1.5; K.DT = 0.5 * (U(rng) + 1.1); K.ALPHA = 0.05 * U(rng);
        Phys<float> Kf{};
        Kf.A = (float)K.A; Kf.B = (float)K.B; Kf.C = (float)K.C; Kf.L = (float)K.L; Kf.LAMBDA = (float)K.LAMBDA;
        Kf.GAMMA = (float)K.GAMMA; Kf.DT = (float)K.DT; Kf.ALPHA = (float)K.ALPHA;
        // two points, inputs exactly representable in float
        auto rf = [&](double s) { return (double)(float)(s * U(rng)); };
        double Q[2][5], u[2][3], ref[2][17];
        QD<double> d[2][5];
        GradU<double> g[2];
        for (int s = 0; s < 2; ++s) {
            for (auto& q : Q[s]) q = rf(0.3);
            for (auto& v : u[s]) v = rf(0.1);
            for (int k = 0; k < 5; ++k) {
                auto& x = d[s][k];
                x.dx = rf(0.1); x.dy = rf(0.1); x.dz = rf(0.1); x.lap = rf(0.1);
                x.d2x = rf(0.1); x.d2y = rf(0.1); x.d2z = rf(0.1);
            }
            g[s] = GradU<double>{rf(0.05), rf(0.05), rf(0.05), rf(0.05), rf(0.05), rf(0.05), rf(0.05), rf(0.05)};
            if (up) reference<true>(K, Q[s], u[s][0], u[s][1], u[s][2], d[s], g[s], ref[s]);
            else reference<false>(K, Q[s], u[s][0], u[s][1], u[s][2], d[s], g[s], ref[s]);
        }
        // the packed form takes unhalved first differences
        auto P2 = [](double a, double b) { return f2((float)a, (float)b); };
        F2 Q2[5], qn[5], pxy[6], pz[3], en[3];
        QD2 d2[5];
        for (int k = 0; k < 5; ++k) {
            Q2[k] = P2(Q[0][k], Q[1][k]);
            d2[k].dx = P2(2 * d[0][k].dx, 2 * d[1][k].dx);
            d2[k].dy = P2(2 * d[0][k].dy, 2 * d[1][k].dy);
            d2[k].dz = P2(2 * d[0][k].dz, 2 * d[1][k].dz);
            d2[k].lap = P2(d[0][k].lap, d[1][k].lap);
            d2[k].d2x = P2(d[0][k].d2x, d[1][k].d2x);
            d2[k].d2y = P2(d[0][k].d2y, d[1][k].d2y);
            d2[k].d2z = P2(d[0][k].d2z, d[1][k].d2z);
        }
        GradU2 g2;
        g2.ux_x = P2(2 * g[0].ux_x, 2 * g[1].ux_x); g2.ux_y = P2(2 * g[0].ux_y, 2 * g[1].ux_y);
        g2.ux_z = P2(2 * g[0].ux_z, 2 * g[1].ux_z); g2.uy_x = P2(2 * g[0].uy_x, 2 * g[1].uy_x);
        g2.uy_y = P2(2 * g[0].uy_y, 2 * g[1].uy_y); g2.uy_z = P2(2 * g[0].uy_z, 2 * g[1].uy_z);
        g2.uz_x = P2(2 * g[0].uz_x, 2 * g[1].uz_x); g2.uz_y = P2(2 * g[0].uz_y, 2 * g[1].uz_y);
        const F2 ux = P2(u[0][0], u[1][0]), uy = P2(u[0][1], u[1][1]), uz = P2(u[0][2], u[1][2]);
        if (up) pointwise_q_pair<true>(Kf, Q2, ux, uy, uz, d2, g2, qn, pxy, pz, en);
        else pointwise_q_pair<false>(Kf, Q2, ux, uy, uz, d2, g2, qn, pxy, pz, en);
        F2 got[17];
        for (int k = 0; k < 5; ++k) got[k] = qn[k];
        for (int k = 0; k < 6; ++k) got[5 + k] = pxy[k];
        for (int k = 0; k < 3; ++k) got[11 + k] = pz[k];
        for (int k = 0; k < 3; ++k) got[14 + k] = en[k];
        for (int i = 0; i < 17; ++i) {
            worst = std::fmax(worst, std::fmax(std::fabs(got[i].v.x - ref[0][i]), std::fabs(got[i].v.y - ref[1][i])));
            scale = std::fmax(scale, std::fmax(std::fabs(ref[0][i]), std::fabs(ref[1][i])));
        }
    }
    std::printf("max abs diff %.3e of max %.3e\n", worst, scale);
    return worst < 2e-5 * scale ? 0 : 1;
}
