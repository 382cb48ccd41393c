// reduce.cuh -- diagnostic reductions on the device: SimIO::Log's sums
// (src/sim_io.cc:83-108), TotalNematicFreeEnergy (src/analysis_fields.h:39-72),
// QtensorToOrderDirector (src/analysis_fields.cc:59-93) and the plaquette
// sign-flip flags of DefectFinder::ComputeWindingNumbers
// (src/analysis/defect_finder.tpp:13-165).
//
// Accumulation is FP64 whatever the field precision.  Pass 1: grid-stride
// loop, warp-shuffle then shared-memory reduction, one partial per block
// (partials[q*G + block]).  Pass 2: one block folds the partials in a fixed
// order, so results are deterministic run to run.
#pragma once

#include "common.cuh"

namespace lbman {

constexpr int kRedThreads = 256;
constexpr int kFlowQ = 8;  // mass px py pz ke e1 e2 | umax2

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

// Block reduction of NQ values (the last NMAX of them by max).  Thread 0
// writes partials[q*gridDim.x + blockIdx.x].
template <int NQ, int NMAX>
__device__ __forceinline__ void block_reduce_store(double (&v)[NQ], double* partials) {
    __shared__ double sh[NQ][kRedThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
        const double r = q < NQ - NMAX ? warp_sum(v[q]) : warp_max(v[q]);
        if (lane == 0) sh[q][warp] = r;
    }
    __syncthreads();
    if (warp == 0) {
#pragma unroll
        for (int q = 0; q < NQ; ++q) {
            double r = lane < (int)(blockDim.x >> 5) ? sh[q][lane] : (q < NQ - NMAX ? 0.0 : -1.0);
            r = q < NQ - NMAX ? warp_sum(r) : warp_max(r);
            if (lane == 0) partials[(size_t)q * gridDim.x + blockIdx.x] = r;
        }
    }
}

template <class R>
__global__ void __launch_bounds__(kRedThreads) flow_reduce_kernel(SimParams P, const R* __restrict__ rho,
                                                                  const R* __restrict__ u,
                                                                  R* __restrict__ upast,
                                                                  double* __restrict__ partials) {
    const int64_t V = P.V;
    double v[kFlowQ] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int64_t c = P.c0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < P.c1;
         c += (int64_t)gridDim.x * blockDim.x) {
        const double r = (double)rho[c];
        const double ux = (double)u[c], uy = (double)u[V + c], uz = (double)u[2 * V + c];
        const double px = (double)upast[c], py = (double)upast[V + c], pz = (double)upast[2 * V + c];
        v[0] += r;
        v[1] += r * ux;
        v[2] += r * uy;
        v[3] += r * uz;
        const double u2 = ux * ux + uy * uy + uz * uz;
        v[4] += 0.5 * r * u2;
        v[5] += (ux - px) * (ux - px) + (uy - py) * (uy - py) + (uz - pz) * (uz - pz);
        v[6] += u2;
        v[7] = fmax(v[7], u2);
        upast[c] = u[c];
        upast[V + c] = u[V + c];
        upast[2 * V + c] = u[2 * V + c];
    }
    block_reduce_store<kFlowQ, 1>(v, partials);
}

// NematicFreeEnergyDensity with the QXoff-clamped 7-point Laplacian.
template <class R>
__global__ void __launch_bounds__(kRedThreads) energy_reduce_kernel(SimParams P, const R* __restrict__ q,
                                                                    double* __restrict__ partials) {
    const int64_t V = P.V;
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    double v[1] = {0.0};
    for (int64_t c = P.c0 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < P.c1;
         c += (int64_t)gridDim.x * blockDim.x) {
        const int z = (int)(c / P.nxy);
        const int rr = (int)(c - (int64_t)z * P.nxy);
        const int y = rr / nx, x = rr - y * nx;
        auto off = [&](int a, int s, int n, int lo, int hi) {
            const int t = a + s;
            if (t < 0) return P.qper[lo] ? t + n : 0;
            if (t >= n) return P.qper[hi] ? t - n : n - 1;
            return t;
        };
        const int xm = off(x, -1, nx, 0, 1), xp = off(x, 1, nx, 0, 1);
        const int ym = off(y, -1, ny, 2, 3), yp = off(y, 1, ny, 2, 3);
        const int zm = off(z, -1, nz, 4, 5), zp = off(z, 1, nz, 4, 5);
        double Q[5], l[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            const R* a = q + k * V;
            auto at = [&](int xx, int yy, int zz) { return (double)a[(int64_t)zz * P.nxy + (int64_t)yy * nx + xx]; };
            Q[k] = (double)a[c];
            l[k] = at(xp, y, z) + at(xm, y, z) + at(x, yp, z) + at(x, ym, z) + at(x, y, zp) + at(x, y, zm) -
                   6.0 * Q[k];
        }
        const double Qxx = Q[0], Qxy = Q[1], Qxz = Q[2], Qyy = Q[3], Qyz = Q[4];
        const double half = (Qxx * Qxx + Qxx * Qyy + Qyy * Qyy + Qxy * Qxy + Qxz * Qxz + Qyz * Qyz);
        const double TrQ2 = 2.0 * half;
        const double k13 = 1.0 / 3.0;
        const double Q2_xx = Qxx * Qxx + Qxy * Qxy + Qxz * Qxz - k13 * TrQ2;
        const double Q2_xy = Qxx * Qxy + Qxy * Qyy + Qxz * Qyz;
        const double Q2_xz = Qxy * Qyz - Qxz * Qyy;
        const double Q2_yy = Qxy * Qxy + Qyy * Qyy + Qyz * Qyz - k13 * TrQ2;
        const double Q2_yz = Qxy * Qxz - Qyz * Qxx;
        const double TrQ3 = 2.0 * Qxx * Q2_xx + 2.0 * Qyy * Q2_yy + Qxx * Q2_yy + Qyy * Q2_xx +
                            2.0 * (Qxy * Q2_xy + Qxz * Q2_xz + Qyz * Q2_yz);
        const double QlQ = 2.0 * Qxx * l[0] + 2.0 * Qyy * l[3] + Qxx * l[3] + Qyy * l[0] +
                           2.0 * (Qxy * l[1] + Qxz * l[2] + Qyz * l[4]);
        v[0] += 0.5 * P.A * TrQ2 + (P.B / 3.0) * TrQ3 + 0.25 * P.C * TrQ2 * TrQ2 - 0.5 * P.L * QlQ;
    }
    block_reduce_store<1, 0>(v, partials);
}

// Scalar order S and director n per cell (closed form, no diagonalisation).
template <class R>
__global__ void __launch_bounds__(kRedThreads) director_kernel(SimParams P, const R* __restrict__ q,
                                                               R* __restrict__ order,
                                                               R* __restrict__ director) {
    const int64_t V = P.V;
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < V; c += (int64_t)gridDim.x * blockDim.x) {
        const double Qxx = q[c], Qxy = q[V + c], Qxz = q[2 * V + c], Qyy = q[3 * V + c], Qyz = q[4 * V + c];
        const double pp = (Qxx * Qxx + Qxx * Qyy + Qyy * Qyy + Qxy * Qxy + Qxz * Qxz + Qyz * Qyz);
        const double qq = (-(Qxx + Qyy) * (Qxx * Qyy - Qxy * Qxy) - Qyy * Qxz * Qxz - Qxx * Qyz * Qyz +
                           2 * Qxy * Qxz * Qyz);
        const double r = 2.0 * sqrt(pp / 3.0);
        double arg = 4 * qq / (r * r * r);
        arg = arg < -1.0 ? -1.0 : (1.0 < arg ? 1.0 : arg);
        const double S = r * cos(1.0 / 3.0 * acos(arg));
        double nx_ = Qxz * (Qyy - S) - Qxy * Qyz;
        double ny_ = Qyz * (Qxx - S) - Qxy * Qxz;
        double nz_ = Qxy * Qxy - (Qxx - S) * (Qyy - S);
        const double ninv = 1.0 / sqrt(nx_ * nx_ + ny_ * ny_ + nz_ * nz_);
        if (order) order[c] = (R)S;
        director[3 * c + 0] = (R)(nx_ * ninv);
        director[3 * c + 1] = (R)(ny_ * ninv);
        director[3 * c + 2] = (R)(nz_ * ninv);
    }
}

template <class R>
__device__ __forceinline__ int plaquette_flip(const R* d1, const R* d2, const R* d3, const R* d4) {
    auto dot = [](const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; };
    const double n1[3] = {(double)d1[0], (double)d1[1], (double)d1[2]};
    double n2[3] = {(double)d2[0], (double)d2[1], (double)d2[2]};
    double n3[3] = {(double)d3[0], (double)d3[1], (double)d3[2]};
    double n4[3] = {(double)d4[0], (double)d4[1], (double)d4[2]};
    if (dot(n1, n2) <= 0.0) { n2[0] = -n2[0]; n2[1] = -n2[1]; n2[2] = -n2[2]; }
    if (dot(n2, n3) <= 0.0) { n3[0] = -n3[0]; n3[1] = -n3[1]; n3[2] = -n3[2]; }
    if (dot(n3, n4) <= 0.0) { n4[0] = -n4[0]; n4[1] = -n4[1]; n4[2] = -n4[2]; }
    return dot(n4, n1) <= 0.0;
}

// Count of flagged plaquettes over the three face families (the periodic
// seam faces are not visited, as in the reference).
template <class R>
__global__ void __launch_bounds__(kRedThreads) defect_count_kernel(SimParams P, const R* __restrict__ dir,
                                                                   double* __restrict__ partials) {
    const int64_t V = P.V;
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    double v[1] = {0.0};
    auto D = [&](int x, int y, int z) { return dir + 3 * ((int64_t)z * P.nxy + (int64_t)y * nx + x); };
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < V; c += (int64_t)gridDim.x * blockDim.x) {
        const int z = (int)(c / P.nxy);
        const int rr = (int)(c - (int64_t)z * P.nxy);
        const int y = rr / nx, x = rr - y * nx;
        int n = 0;
        if (y < ny - 1 && z < nz - 1) n += plaquette_flip<R>(D(x, y, z), D(x, y + 1, z), D(x, y + 1, z + 1), D(x, y, z + 1));
        if (x < nx - 1 && z < nz - 1) n += plaquette_flip<R>(D(x, y, z), D(x + 1, y, z), D(x + 1, y, z + 1), D(x, y, z + 1));
        if (x < nx - 1 && y < ny - 1) n += plaquette_flip<R>(D(x, y, z), D(x + 1, y, z), D(x + 1, y + 1, z), D(x, y + 1, z));
        v[0] += n;
    }
    block_reduce_store<1, 0>(v, partials);
}

// Plaquette flags of the three face families in the reference's DefectFields
// layout (src/analysis/defect_fields.h:16-29): def_x nx*(ny-1)*(nz-1), then
// def_y (nx-1)*ny*(nz-1), then def_z (nx-1)*(ny-1)*nz, each x fastest.
template <class R>
__global__ void __launch_bounds__(kRedThreads) defect_flags_kernel(SimParams P, const R* __restrict__ dir,
                                                                   uint8_t* __restrict__ flags) {
    const int64_t V = P.V;
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const int64_t nfx = (int64_t)nx * (ny - 1) * (nz - 1), nfy = (int64_t)(nx - 1) * ny * (nz - 1);
    auto D = [&](int x, int y, int z) { return dir + 3 * ((int64_t)z * P.nxy + (int64_t)y * nx + x); };
    for (int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; c < V; c += (int64_t)gridDim.x * blockDim.x) {
        const int z = (int)(c / P.nxy);
        const int rr = (int)(c - (int64_t)z * P.nxy);
        const int y = rr / nx, x = rr - y * nx;
        if (y < ny - 1 && z < nz - 1)
            flags[((int64_t)z * (ny - 1) + y) * nx + x] =
                (uint8_t)plaquette_flip<R>(D(x, y, z), D(x, y + 1, z), D(x, y + 1, z + 1), D(x, y, z + 1));
        if (x < nx - 1 && z < nz - 1)
            flags[nfx + ((int64_t)z * ny + y) * (nx - 1) + x] =
                (uint8_t)plaquette_flip<R>(D(x, y, z), D(x + 1, y, z), D(x + 1, y, z + 1), D(x, y, z + 1));
        if (x < nx - 1 && y < ny - 1)
            flags[nfx + nfy + ((int64_t)z * (ny - 1) + y) * (nx - 1) + x] =
                (uint8_t)plaquette_flip<R>(D(x, y, z), D(x + 1, y, z), D(x + 1, y + 1, z), D(x, y + 1, z));
    }
}

// Pass 2: fold G partials of NQ quantities (the last nmax by max) in order.
static __global__ void __launch_bounds__(1024) fold_partials_kernel(const double* __restrict__ partials, int G,
                                                             int nq, int nmax, double* __restrict__ out) {
    __shared__ double sh[32];
    for (int q = 0; q < nq; ++q) {
        const bool is_max = q >= nq - nmax;
        double acc = is_max ? -1.0 : 0.0;
        for (int b = threadIdx.x; b < G; b += blockDim.x) {
            const double x = partials[(size_t)q * G + b];
            acc = is_max ? fmax(acc, x) : acc + x;
        }
        acc = is_max ? warp_max(acc) : warp_sum(acc);
        if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = acc;
        __syncthreads();
        if (threadIdx.x < 32) {
            double r = threadIdx.x < (blockDim.x >> 5) ? sh[threadIdx.x] : (is_max ? -1.0 : 0.0);
            r = is_max ? warp_max(r) : warp_sum(r);
            if (threadIdx.x == 0) out[q] = r;
        }
        __syncthreads();
    }
}

}  // namespace lbman
