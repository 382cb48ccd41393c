// lbm.cuh -- D3Q15 collide + stream + wall rules (LbmSolver::
// LatticeBoltzmannStep, src/lbm_solver.tpp:65-199) as a pull-scheme kernel.
//
// The reference pushes: each cell collides and scatters f* to its
// neighbours, with HandleBoundaryPoint (src/boundary_handler.h:403-426)
// writing reflected populations back at the source cell.  Here every cell
// gathers instead: the population arriving in direction j at cell c is
//   * f*[c - e_j][j] when c - e_j is inside the box (periodic axes wrap);
//   * otherwise, for each wall axis A that c - e_j leaves, the reference's
//     rule on that wall would have written slot j at c from direction
//     i_A = opp(j) (no-slip / moving wall) or spec_A(j) (specular);
//     the reference applies those writes in (i, axis) order, so the last one
//     (largest i, then largest axis) is the value that survives.  A moving
//     wall adds 6 rho w_j (e_j . U_wall) with rho of cell c from the step
//     that produced f*.
// Each population is therefore read once and written once per step, fully
// coalesced along x.  The stored state is post-collision (f*); the first
// step after an upload reads the pre-collision populations in place.
//
// Storage precision S (double / float / half) and compute precision R are
// template parameters.  DEV stores populations as deviations f_i - w_i rho0
// (rho0 = kDensity), which keeps FP32/FP16 rounding relative to the small
// non-equilibrium part.
#pragma once

#include "common.cuh"

namespace lbman {

// Unsigned division by a run-time constant (round-up multiply-shift), exact
// for numerators below 2^31.
struct FastDiv {
    uint32_t d, m, s;
};
inline FastDiv make_fastdiv(uint32_t d) {
    FastDiv f;
    f.d = d;
    uint32_t l = 0;
    while ((1ull << l) < d) ++l;
    f.s = l;
    f.m = (uint32_t)((((1ull << l) - d) << 32) / d + 1);
    return f;
}
__device__ __forceinline__ uint32_t fdiv(uint32_t n, const FastDiv& f) {
    return (__umulhi(n, f.m) + n) >> f.s;
}

template <class R>
__device__ __forceinline__ R sgn_term(int e, R v) {
    return e > 0 ? v : -v;
}
// (a*ex + b*ey) + c*ez with the zero terms left out: the same value as the
// reference's Vec3::Dot with integer-valued e (src/physics_helpers.h:29-31).
template <class R>
__device__ __forceinline__ R edot(int ex, int ey, int ez, R a, R b, R c) {
    R s = R(0);
    bool has = false;
    if (ex) { s = sgn_term(ex, a); has = true; }
    if (ey) { const R t = sgn_term(ey, b); s = has ? s + t : t; has = true; }
    if (ez) { const R t = sgn_term(ez, c); s = has ? s + t : t; has = true; }
    return s;
}

struct CellPos {
    int x, y, z;
};

__device__ __forceinline__ bool touches_moving(const SimParams& P, int x, int y, int z) {
    return (x == 0 && P.face[0].ubc == U_MOVING) || (x == P.nx - 1 && P.face[1].ubc == U_MOVING) ||
           (y == 0 && P.face[2].ubc == U_MOVING) || (y == P.ny - 1 && P.face[3].ubc == U_MOVING) ||
           (z == 0 && P.face[4].ubc == U_MOVING) || (z == P.nz - 1 && P.face[5].ubc == U_MOVING);
}

// Gather the 15 pre-collision populations of cell c from the post-collision
// buffer fin (see the rule above).
template <class R, class S>
__device__ __forceinline__ void gather(const SimParams& P, const S* __restrict__ fin, int64_t c,
                                       CellPos q, R rho_prev, R f[15]) {
    const int64_t V = P.V;
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const bool interior = q.x > 0 && q.x < nx - 1 && q.y > 0 && q.y < ny - 1 && q.z > 0 && q.z < nz - 1;
    if (interior) {
#pragma unroll
        for (int j = 0; j < 15; ++j)
            f[j] = Store<S>::ld(fin + j * V + c - (ex_(j) + (int64_t)ey_(j) * nx + (int64_t)ez_(j) * P.nxy));
        return;
    }
#pragma unroll
    for (int j = 0; j < 15; ++j) {
        int sx = q.x - ex_(j), sy = q.y - ey_(j), sz = q.z - ez_(j);
        int cross = 0, fxs = 0, fys = 0, fzs = 0;
        if (sx < 0) { if (P.uper[0]) sx += nx; else { cross |= 1; fxs = 0; } }
        else if (sx >= nx) { if (P.uper[1]) sx -= nx; else { cross |= 1; fxs = 1; } }
        if (sy < 0) { if (P.uper[2]) sy += ny; else { cross |= 2; fys = 2; } }
        else if (sy >= ny) { if (P.uper[3]) sy -= ny; else { cross |= 2; fys = 3; } }
        if (sz < 0) { if (P.uper[4]) sz += nz; else { cross |= 4; fzs = 4; } }
        else if (sz >= nz) { if (P.uper[5]) sz -= nz; else { cross |= 4; fzs = 5; } }
        if (!cross) {
            f[j] = Store<S>::ld(fin + j * V + (int64_t)sz * P.nxy + (int64_t)sy * nx + sx);
            continue;
        }
        int bi = -1, bf = 0;
        if (cross & 1) { const int i = P.face[fxs].ubc == U_SPECULAR ? spec_(0, j) : opp_(j); if (i >= bi) { bi = i; bf = fxs; } }
        if (cross & 2) { const int i = P.face[fys].ubc == U_SPECULAR ? spec_(1, j) : opp_(j); if (i >= bi) { bi = i; bf = fys; } }
        if (cross & 4) { const int i = P.face[fzs].ubc == U_SPECULAR ? spec_(2, j) : opp_(j); if (i >= bi) { bi = i; bf = fzs; } }
        R v = Store<S>::ld(fin + (int64_t)bi * V + c);
        if (P.face[bf].ubc == U_MOVING) {
            const R dot = R(ex_(j)) * R(P.face[bf].uw[0]) + R(ey_(j)) * R(P.face[bf].uw[1]) +
                          R(ez_(j)) * R(P.face[bf].uw[2]);
            v = v + R(6.0) * rho_prev * w_<R>(j) * dot;
        }
        f[j] = v;
    }
}

// Moments, equilibrium, Guo forcing and BGK relaxation of one cell
// (src/physics_helpers.h:69-129); f is overwritten with f*.
template <class R, bool DEV>
__device__ __forceinline__ void collide(const SimParams& P, R f[15], R Fx, R Fy, R Fz, R& rho, R& ux,
                                        R& uy, R& uz) {
    const R DT = R(P.DT);
    R s = f[0];
#pragma unroll
    for (int j = 1; j < 15; ++j) s = s + f[j];
    R jx = R(0), jy = R(0), jz = R(0);
    bool hx = false, hy = false, hz = false;
#pragma unroll
    for (int j = 0; j < 15; ++j) {
        if (ex_(j)) { const R t = sgn_term(ex_(j), f[j]); jx = hx ? jx + t : t; hx = true; }
        if (ey_(j)) { const R t = sgn_term(ey_(j), f[j]); jy = hy ? jy + t : t; hy = true; }
        if (ez_(j)) { const R t = sgn_term(ez_(j), f[j]); jz = hz ? jz + t : t; hz = true; }
    }
    const R rho0 = R(P.kDensity);
    rho = DEV ? rho0 + s : s;  // DEV: s is the density deviation
    ux = (jx + R(0.5) * Fx * DT) / rho;
    uy = (jy + R(0.5) * Fy * DT) / rho;
    uz = (jz + R(0.5) * Fz * DT) / rho;
    const R uF = ux * Fx + uy * Fy + uz * Fz;
    const R u2 = ux * ux + uy * uy + uz * uz;
    const R om = R(P.omega), omp = R(P.omega_prime), omf = R(P.omega_forcing);
#pragma unroll
    for (int j = 0; j < 15; ++j) {
        const R w = w_<R>(j);
        const R ue = edot<R>(ex_(j), ey_(j), ez_(j), ux, uy, uz);
        const R eF = edot<R>(ex_(j), ey_(j), ez_(j), Fx, Fy, Fz);
        const R poly = R(1.0) + R(3.0) * ue + R(4.5) * ue * ue - R(1.5) * u2;
        // DEV: f_eq - w rho0 = w (rho - rho0) + w rho (poly - 1)
        const R feq = DEV ? w * (s + rho * (poly - R(1.0))) : w * rho * poly;
        const R forcing = omf * w * (R(3.0) * eF - R(3.0) * uF + R(9.0) * ue * eF);
        f[j] = om * f[j] + omp * feq + DT * forcing;
    }
}

// One LBM step.  FIRST: fin holds pre-collision populations (just uploaded).
template <class R, class S, bool DEV, bool FIRST>
__global__ void __launch_bounds__(256) lbm_kernel(SimParams P, FastDiv dnx, FastDiv dnxy,
                                                  const S* __restrict__ fin, S* __restrict__ fout,
                                                  const R* __restrict__ F, R* __restrict__ rho_buf,
                                                  R* __restrict__ uout, int write_rho_all) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.V) return;
    const int64_t V = P.V;
    CellPos q;
    q.z = (int)fdiv((uint32_t)c, dnxy);
    const uint32_t r = (uint32_t)(c - (int64_t)q.z * P.nxy);
    q.y = (int)fdiv(r, dnx);
    q.x = (int)(r - (uint32_t)q.y * (uint32_t)P.nx);
    const bool mv = P.moving_any && touches_moving(P, q.x, q.y, q.z);
    R f[15];
    if (FIRST) {
#pragma unroll
        for (int j = 0; j < 15; ++j) f[j] = Store<S>::ld(fin + j * V + c);
    } else {
        const R rp = mv ? rho_buf[c] : R(0);
        gather<R, S>(P, fin, c, q, rp, f);
    }
    R rho, ux, uy, uz;
    collide<R, DEV>(P, f, F[c], F[V + c], F[2 * V + c], rho, ux, uy, uz);
#pragma unroll
    for (int j = 0; j < 15; ++j) Store<S>::st(fout + j * V + c, f[j]);
    uout[c] = ux;
    uout[V + c] = uy;
    uout[2 * V + c] = uz;
    if (write_rho_all || mv) rho_buf[c] = rho;
}

// Pre-collision populations from the stored post-collision ones (for a
// download of f): the gather alone.
template <class R, class S>
__global__ void __launch_bounds__(256) stream_only_kernel(SimParams P, FastDiv dnx, FastDiv dnxy,
                                                          const S* __restrict__ fin,
                                                          S* __restrict__ fout,
                                                          const R* __restrict__ rho_buf) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.V) return;
    CellPos q;
    q.z = (int)fdiv((uint32_t)c, dnxy);
    const uint32_t r = (uint32_t)(c - (int64_t)q.z * P.nxy);
    q.y = (int)fdiv(r, dnx);
    q.x = (int)(r - (uint32_t)q.y * (uint32_t)P.nx);
    const bool mv = P.moving_any && touches_moving(P, q.x, q.y, q.z);
    R f[15];
    gather<R, S>(P, fin, c, q, mv ? rho_buf[c] : R(0), f);
#pragma unroll
    for (int j = 0; j < 15; ++j) Store<S>::st(fout + j * P.V + c, f[j]);
}

// f = f_eq(rho, u) (LbmSolver::Initialize, src/lbm_solver.tpp:35-62).
template <class R, class S, bool DEV>
__global__ void __launch_bounds__(256) feq_init_kernel(SimParams P, const R* __restrict__ rho,
                                                       const R* __restrict__ u, S* __restrict__ f) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.V) return;
    const int64_t V = P.V;
    const R r = rho[c], ux = u[c], uy = u[V + c], uz = u[2 * V + c];
    const R u2 = ux * ux + uy * uy + uz * uz;
    const R rho0 = R(P.kDensity);
#pragma unroll
    for (int j = 0; j < 15; ++j) {
        const R w = w_<R>(j);
        const R ue = edot<R>(ex_(j), ey_(j), ez_(j), ux, uy, uz);
        const R poly = R(1.0) + R(3.0) * ue + R(4.5) * ue * ue - R(1.5) * u2;
        const R v = DEV ? w * ((r - rho0) + r * (poly - R(1.0))) : w * r * poly;
        Store<S>::st(f + j * V + c, v);
    }
}

}  // namespace lbman
