// common.cuh -- device-side parameters, D3Q15 tables and boundary helpers
// shared by every kernel of the sm_100a implementation.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace lbman {

enum : int { Q_PERIODIC = 0, Q_NEUMANN = 1, Q_ANCHORING = 2 };
enum : int { U_PERIODIC = 0, U_NOSLIP = 1, U_MOVING = 2, U_SPECULAR = 3 };

// One face of the box at run time: WallSpec<QBC, UBC> lowered from the
// reference's type tags (src/boundary.h:72-76).  The anchoring target Q is
// evaluated on the host once (AnchoredQ, src/boundary_handler.h:232-251) so
// every kernel and the CPU oracle use the same bits.
struct Face {
    int qbc, ubc;
    double anchor[5];
    double uw[3];
};

// params.h + SimBC at run time.  Passed by value to every kernel.
struct SimParams {
    int nx, ny, nz;
    int64_t V, nxy;
    double DT, kDensity, L, A, B, C, LAMBDA, GAMMA, ALPHA, MU;
    double omega, omega_prime, omega_forcing;
    int upwind;
    Face face[6];          // XLo, XHi, YLo, YHi, ZLo, ZHi
    int qper[6], uper[6];  // face tag is Periodic (Q / velocity)
    int moving_any;        // some face is a MovingWall
};

// z-marching tile of the Q+force kernel (runtime shape, chosen by the autotuner).
struct QTile {
    int tcx, tcy;  // output cells per plane
    int zc;        // z planes per block
};

// D3Q15 (src/lattice_stencil.h:42-76): velocities, weights, opposite and
// specular partners.  Values are compile-time constants so unrolled loops
// fold them.
__host__ __device__ constexpr int ex_(int i) {
    constexpr int t[15] = {0, 1, 0, -1, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
    return t[i];
}
__host__ __device__ constexpr int ey_(int i) {
    constexpr int t[15] = {0, 0, 1, 0, -1, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
    return t[i];
}
__host__ __device__ constexpr int ez_(int i) {
    constexpr int t[15] = {0, 0, 0, 0, 0, 1, -1, 1, 1, 1, 1, -1, -1, -1, -1};
    return t[i];
}
__host__ __device__ constexpr int opp_(int i) {
    constexpr int t[15] = {0, 3, 4, 1, 2, 6, 5, 13, 14, 11, 12, 9, 10, 7, 8};
    return t[i];
}
__host__ __device__ constexpr int spec_(int ax, int i) {
    constexpr int t[3][15] = {{0, 3, 2, 1, 4, 5, 6, 8, 7, 10, 9, 12, 11, 14, 13},
                              {0, 1, 4, 3, 2, 5, 6, 10, 9, 8, 7, 14, 13, 12, 11},
                              {0, 1, 2, 3, 4, 6, 5, 11, 12, 13, 14, 7, 8, 9, 10}};
    return t[ax][i];
}
template <class R>
__host__ __device__ constexpr R w_(int i) {
    return i == 0 ? R(2.0 / 9) : (i < 7 ? R(1.0 / 9) : R(1.0 / 72));
}

// Storage conversions for populations.
template <class S> struct Store;
template <> struct Store<double> {
    __device__ static double ld(const double* p) { return __ldg(p); }
    __device__ static void st(double* p, double v) { *p = v; }
};
template <> struct Store<float> {
    __device__ static float ld(const float* p) { return __ldg(p); }
    __device__ static void st(float* p, float v) { *p = v; }
};
template <> struct Store<__half> {
    __device__ static float ld(const __half* p) { return __half2float(__ldg(p)); }
    __device__ static void st(__half* p, float v) { *p = __float2half_rn(v); }
};

__host__ __device__ inline int wrap_coord(int a, int n) {
    if (a >= 0 && a < n) return a;
    int r = a % n;
    return r < 0 ? r + n : r;
}

}  // namespace lbman
