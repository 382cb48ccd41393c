// init.cuh -- seeded initial condition on the device: rho = kDensity, u = 0,
// Q = S0 (n n^T - I/3) with n uniform on the sphere per cell plus
// N(0, sigma^2) on each of the 5 stored components.  Counter based
// (splitmix64 of the seed and the cell index), so the field does not depend
// on the launch shape; the same generator runs on the host in the test
// oracle (there with the host libm, so values agree to a few ulp).
#pragma once

#include "common.cuh"

namespace lbman {

__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

__device__ __forceinline__ double uniform01(uint64_t key, uint64_t cell, uint64_t k) {
    const uint64_t h = splitmix64(key + cell * 16u + k);
    return ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

template <class R>
__global__ void __launch_bounds__(256) seeded_init_kernel(SimParams P, uint64_t key, double S0, double sigma,
                                                          R* __restrict__ rho, R* __restrict__ u,
                                                          R* __restrict__ q, R* __restrict__ F) {
    const int64_t c = P.c0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.c1) return;
    const int64_t V = P.V;
    const uint64_t gc = (uint64_t)(c + P.gbase);  // index in the whole box
    const double two_pi = 6.283185307179586476925286766559;
    const double ct = 2.0 * uniform01(key, gc, 0) - 1.0;
    const double ph = two_pi * uniform01(key, gc, 1);
    const double st = sqrt(fmax(0.0, 1.0 - ct * ct));
    const double n0 = st * cos(ph), n1 = st * sin(ph), n2 = ct;
    double g[6];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double r = sqrt(-2.0 * log(uniform01(key, gc, 2 + 2 * k)));
        const double t = two_pi * uniform01(key, gc, 3 + 2 * k);
        g[2 * k] = r * cos(t);
        g[2 * k + 1] = r * sin(t);
    }
    q[c] = (R)(S0 * (n0 * n0 - 1.0 / 3.0) + sigma * g[0]);
    q[V + c] = (R)(S0 * (n0 * n1) + sigma * g[1]);
    q[2 * V + c] = (R)(S0 * (n0 * n2) + sigma * g[2]);
    q[3 * V + c] = (R)(S0 * (n1 * n1 - 1.0 / 3.0) + sigma * g[3]);
    q[4 * V + c] = (R)(S0 * (n1 * n2) + sigma * g[4]);
    rho[c] = (R)P.kDensity;
    u[c] = u[V + c] = u[2 * V + c] = R(0);
    F[c] = F[V + c] = F[2 * V + c] = R(0);
}

}  // namespace lbman
