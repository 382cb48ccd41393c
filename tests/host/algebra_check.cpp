// Compiles the device physics (physics.cuh) as host C++ and checks the FP32
// right-hand side (pointwise_q_mat: unhalved differences, QB + (QB)^T and
// QH +/- HQ forms) against the reference-ordered one (pointwise_q), both
// evaluated in double, on random states, centred and upwind.  Exit 0 iff they
// agree to 1e-12 of the largest output.
#define __device__
#define __host__
#define __forceinline__ inline
#define __global__
#include <cstdio>
#include <cmath>
#include <random>
#include "common.cuh"
#include "physics.cuh"
using namespace lbman;
int main() {
    std::mt19937_64 rng(1);
    std::uniform_real_distribution<double> U(-1, 1);
    double worst = 0, scale = 0;
    for (int trial = 0; trial < 2000; ++trial) {
        Phys<double> K{};
        K.A = 0.5 * (U(rng) + 1); K.B = U(rng); K.C = 0.5 * (U(rng) + 1); K.L = 0.1 * (U(rng) + 1);
        K.LAMBDA = U(rng); K.GAMMA = U(rng) + 1.5; K.DT = 0.5 * (U(rng) + 1.1);
        double Q[5]; for (auto& q : Q) q = 0.3 * U(rng);
        double ux = 0.1 * U(rng), uy = 0.1 * U(rng), uz = 0.1 * U(rng);
        QD<double> d[5], d2[5];
        for (int k = 0; k < 5; ++k) {
            auto& x = d[k];
            x.dx = 0.1 * U(rng); x.dy = 0.1 * U(rng); x.dz = 0.1 * U(rng); x.lap = 0.1 * U(rng);
            x.d2x = 0.1 * U(rng); x.d2y = 0.1 * U(rng); x.d2z = 0.1 * U(rng);
            d2[k] = x; d2[k].dx = 2 * x.dx; d2[k].dy = 2 * x.dy; d2[k].dz = 2 * x.dz;
        }
        GradU<double> g{0.05 * U(rng), 0.05 * U(rng), 0.05 * U(rng), 0.05 * U(rng), 0.05 * U(rng), 0.05 * U(rng), 0.05 * U(rng), 0.05 * U(rng)};
        GradU<double> g2{2 * g.ux_x, 2 * g.ux_y, 2 * g.ux_z, 2 * g.uy_x, 2 * g.uy_y, 2 * g.uy_z, 2 * g.uz_x, 2 * g.uz_y};
        double a[16], b[16];
        for (int up = 0; up < 2; ++up) {
            if (up) {
                pointwise_q<double, true>(K, Q, ux, uy, uz, d, g, a, a + 5, a + 10, a + 13);
                pointwise_q_mat<double, true>(K, Q, ux, uy, uz, d2, g2, b, b + 5, b + 10, b + 13);
            } else {
                pointwise_q<double, false>(K, Q, ux, uy, uz, d, g, a, a + 5, a + 10, a + 13);
                pointwise_q_mat<double, false>(K, Q, ux, uy, uz, d2, g2, b, b + 5, b + 10, b + 13);
            }
            for (int i = 0; i < 16; ++i) { worst = std::fmax(worst, std::fabs(a[i] - b[i])); scale = std::fmax(scale, std::fabs(a[i])); }
        }
    }
    std::printf("max abs diff %.3e of max %.3e\n", worst, scale);
    return worst < 1e-12 * scale ? 0 : 1;
}
