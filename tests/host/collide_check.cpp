// Compiles the D3Q15 collision (lbm.cuh) as host C++ and checks the paired
// relaxation of the FP32 instantiations (relax_pairs) against the
// direction-by-direction form (collide with R = double), both in double, on
// random populations and forces, with deviation storage and without.  Exit 0
// iff they agree to 1e-13 of the largest population, and the whole FP32
// collision (pairwise moments included) agrees with it to FP32 rounding.
#define __device__
#define __host__
#define __forceinline__ inline
#define __global__
#define __launch_bounds__(...)
#define __grid_constant__
#include <cstdint>
inline uint32_t __umulhi(uint32_t a, uint32_t b) { return (uint32_t)(((uint64_t)a * b) >> 32); }
struct HostDim3 { unsigned x = 0, y = 0, z = 0; };
static HostDim3 blockIdx, blockDim, threadIdx;  // the kernels are compiled, never run
#include <cmath>
#include <cstdio>
#include <random>
#include "common.cuh"
#include "lbm.cuh"
using namespace lbman;

static double worst_f32 = 0;

template <bool DEV>
double run(std::mt19937_64& rng) {
    std::uniform_real_distribution<double> U(-1, 1);
    Phys<double> K{};
    K.DT = 1.0;
    K.kDensity = 1.0;
    const double tau = 0.6 + 0.5 * (U(rng) + 1);
    K.omega = 1.0 - 1.0 / tau;
    K.omega_prime = 1.0 / tau;
    K.omega_forcing = 1.0 - 0.5 / tau;
    double worst = 0;
    for (int trial = 0; trial < 2000; ++trial) {
        double f[15], g[15], g0[15];
        for (int j = 0; j < 15; ++j) {
            const double w = w_<double>(j);
            f[j] = (DEV ? 0.0 : w) + 0.01 * w * U(rng);
            g[j] = g0[j] = f[j];
        }
        const double Fx = 1e-3 * U(rng), Fy = 1e-3 * U(rng), Fz = 1e-3 * U(rng);
        double rho, ux, uy, uz;
        collide<double, DEV>(K, f, Fx, Fy, Fz, rho, ux, uy, uz);  // reference order
        // the paired form on the same moments
        double s = g[0];
        for (int j = 1; j < 15; ++j) s += g[j];
        const double uF = ux * Fx + uy * Fy + uz * Fz, u2 = ux * ux + uy * uy + uz * uz;
        relax_pairs<double, DEV>(K.omega, K.omega_prime, K.omega_forcing, K.DT, s, rho, ux, uy, uz, Fx, Fy, Fz, uF,
                                 u2, g);
        for (int j = 0; j < 15; ++j) worst = std::fmax(worst, std::fabs(f[j] - g[j]));
        // the whole FP32 instantiation (pairwise moments + paired relaxation)
        // against the double reference, within FP32 rounding
        Phys<float> Kf{};
        Kf.DT = (float)K.DT; Kf.kDensity = (float)K.kDensity; Kf.omega = (float)K.omega;
        Kf.omega_prime = (float)K.omega_prime; Kf.omega_forcing = (float)K.omega_forcing;
        float h[15];
        for (int j = 0; j < 15; ++j) h[j] = (float)g0[j];
        float rf, uxf, uyf, uzf;
        collide<float, DEV>(Kf, h, (float)Fx, (float)Fy, (float)Fz, rf, uxf, uyf, uzf);
        double scale = 0;
        for (int j = 0; j < 15; ++j) scale = std::fmax(scale, std::fabs(f[j]));
        for (int j = 0; j < 15; ++j) worst_f32 = std::fmax(worst_f32, std::fabs(h[j] - f[j]) / scale);
    }
    return worst;
}

int main() {
    std::mt19937_64 rng(3);
    const double a = run<true>(rng), b = run<false>(rng);
    std::printf("max abs diff: deviation %.3e, plain %.3e; FP32 collide max rel diff %.3e\n", a, b, worst_f32);
    return (a < 1e-15 && b < 1e-13 && worst_f32 < 1e-5) ? 0 : 1;
}
