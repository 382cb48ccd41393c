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

// Physical constants in compute precision R (the FP32 copy is rounded once
// on the host, so kernels do no double-to-float conversions).
template <class R>
struct Phys {
    R DT, kDensity, L, A, B, C, LAMBDA, GAMMA, ALPHA, MU;
    R omega, omega_prime, omega_forcing;
    R anchor[6][5];
    R uw[6][3];
};

// params.h + SimBC at run time.  Passed by value to every kernel.
struct SimParams {
    int nx, ny, nz;
    int64_t V, nxy;
    // The planes [zlo, zhi) and cells [c0, c1) a step updates: the whole box,
    // or the owned planes of a z-slab allocated with ghost planes on both
    // sides (the z axis is then periodic in the kernels' view and never
    // wraps, because every neighbour of an owned plane is allocated).  gbase
    // maps a cell index to its index in the whole box.
    int zlo, zhi;
    int64_t c0, c1, gbase;
    double DT, kDensity, L, A, B, C, LAMBDA, GAMMA, ALPHA, MU;
    double omega, omega_prime, omega_forcing;
    int upwind;
    Face face[6];          // XLo, XHi, YLo, YHi, ZLo, ZHi
    int qper[6], uper[6];  // face tag is Periodic (Q / velocity)
    int moving_any;        // some face is a MovingWall
    Phys<double> pd;       // the constants above, per compute precision; kernels
    Phys<float> pf;        // read them in place from the parameter space
};

static_assert(sizeof(SimParams) % 4 == 0, "copied to shared memory as 32-bit words");

// Constants of precision R, referenced inside the kernel's (grid-constant)
// parameter struct, so dynamic indexing needs no local copy.
template <class R>
__host__ __device__ inline const Phys<R>& phys_ref(const SimParams& P);
template <>
__host__ __device__ inline const Phys<float>& phys_ref<float>(const SimParams& P) {
    return P.pf;
}
template <>
__host__ __device__ inline const Phys<double>& phys_ref<double>(const SimParams& P) {
    return P.pd;
}

// Fills P.pd / P.pf from the double fields (host side, once per solver).
template <class R>
inline void fill_phys(const SimParams& P, Phys<R>& k) {
    k.DT = (R)P.DT; k.kDensity = (R)P.kDensity; k.L = (R)P.L; k.A = (R)P.A;
    k.B = (R)P.B; k.C = (R)P.C; k.LAMBDA = (R)P.LAMBDA; k.GAMMA = (R)P.GAMMA;
    k.ALPHA = (R)P.ALPHA; k.MU = (R)P.MU; k.omega = (R)P.omega;
    k.omega_prime = (R)P.omega_prime; k.omega_forcing = (R)P.omega_forcing;
    for (int f = 0; f < 6; ++f) {
        for (int c = 0; c < 5; ++c) k.anchor[f][c] = (R)P.face[f].anchor[c];
        for (int c = 0; c < 3; ++c) k.uw[f][c] = (R)P.face[f].uw[c];
    }
}
inline void fill_float_phys(SimParams& P) {
    fill_phys<double>(P, P.pd);
    fill_phys<float>(P, P.pf);
}

// z-marching tile of the Q+force kernel (runtime shape, chosen by the autotuner).
struct QTile {
    int tcx, tcy;  // output cells per plane
    int zc;        // z planes per block
    int pair = 0;  // FP32 Q+force kernel with two points per thread (qpair.cuh)
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
// ld = raw load + widen; the split form lets a gather issue every load before
// the first conversion waits on one.
template <> struct Store<double> {
    __device__ static double ld(const double* p) { return __ldg(p); }
    __device__ static double raw(const double* p) { return __ldg(p); }
    __device__ static double widen(double v) { return v; }
    __device__ static void st(double* p, double v) { *p = v; }
};
template <> struct Store<float> {
    __device__ static float ld(const float* p) { return __ldg(p); }
    __device__ static float raw(const float* p) { return __ldg(p); }
    __device__ static float widen(float v) { return v; }
    __device__ static void st(float* p, float v) { *p = v; }
};
template <> struct Store<__half> {
    __device__ static float ld(const __half* p) { return __half2float(__ldg(p)); }
    __device__ static __half raw(const __half* p) { return __ldg(p); }
    __device__ static float widen(__half v) { return __half2float(v); }
    __device__ static void st(__half* p, float v) { *p = __float2half_rn(v); }
};

__host__ __device__ inline int wrap_coord(int a, int n) {
    if (a >= 0 && a < n) return a;
    int r = a % n;
    return r < 0 ? r + n : r;
}

}  // namespace lbman
