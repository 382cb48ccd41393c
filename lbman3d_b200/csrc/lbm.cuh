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

// The direction whose post-collision value at this cell the reference's
// wall rules leave in slot j when c - e_j lies beyond the crossed walls
// (cx, cy, cz): per crossed axis the candidate opp(j) (no-slip / moving) or
// spec_A(j) (specular); the largest wins, ties to the later axis.  *face, if
// given, receives the winning wall.
__device__ __forceinline__ int wall_source(const SimParams& P, int j, bool cx, bool cy, bool cz, int* face) {
    const int fxs = ex_(j) > 0 ? 0 : 1, fys = ey_(j) > 0 ? 2 : 3, fzs = ez_(j) > 0 ? 4 : 5;
    int bi = -1, bf = 0;
    if (cx) { const int i = P.face[fxs].ubc == U_SPECULAR ? spec_(0, j) : opp_(j); if (i >= bi) { bi = i; bf = fxs; } }
    if (cy) { const int i = P.face[fys].ubc == U_SPECULAR ? spec_(1, j) : opp_(j); if (i >= bi) { bi = i; bf = fys; } }
    if (cz) { const int i = P.face[fzs].ubc == U_SPECULAR ? spec_(2, j) : opp_(j); if (i >= bi) { bi = i; bf = fzs; } }
    if (face) *face = bf;
    return bi;
}

// Gather the 15 pre-collision populations of cell c from the post-collision
// buffer fin (see the rule above).  WALLS = false: every velocity axis is
// periodic (wrap only, no wall logic compiled in).
// I: index type of the population offsets -- int when 15 V < 2^31 (the
// launcher checks), so addresses take 32-bit arithmetic.
template <class R, class S, bool WALLS = true, class I = int64_t>
__device__ __forceinline__ void gather(const SimParams& P, const Phys<R>& K, const S* __restrict__ fin,
                                       I c, CellPos q, R rho_prev, R f[15]) {
    const I V = (I)P.V;
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    // Offsets of the source cell c - e along each axis for e = +1 / -1, with
    // the periodic wrap folded in, and whether that source lies beyond a wall
    // (velocity tags are periodic on both faces of an axis or on neither).
    const bool lox = q.x == 0, hix = q.x == nx - 1, loy = q.y == 0, hiy = q.y == ny - 1;
    const bool loz = q.z == 0, hiz = q.z == nz - 1;
    const I nxy = (I)P.nxy;
    const I ox_m = lox ? (I)(nx - 1) : (I)-1, ox_p = hix ? (I)(1 - nx) : (I)1;
    const I oy_m = loy ? (I)(ny - 1) * nx : -(I)nx;
    const I oy_p = hiy ? -(I)(ny - 1) * nx : (I)nx;
    const I oz_m = loz ? (I)(nz - 1) * nxy : -nxy;
    const I oz_p = hiz ? -(I)(nz - 1) * nxy : nxy;
    const bool wx = !P.uper[0], wy = !P.uper[2], wz = !P.uper[4];
    // Pass 1 issues the 15 loads (raw storage values), pass 2 widens them,
    // pass 3 adds the moving-wall term; no load waits inside pass 1.
    S raw[15];
#pragma unroll
    for (int j = 0; j < 15; ++j) {
        // source = c - e_j: e = +1 looks at the -1 neighbour
        const I off = (ex_(j) > 0 ? ox_m : ex_(j) < 0 ? ox_p : (I)0) +
                      (ey_(j) > 0 ? oy_m : ey_(j) < 0 ? oy_p : (I)0) + (ez_(j) > 0 ? oz_m : ez_(j) < 0 ? oz_p : (I)0);
        if constexpr (!WALLS) {
            raw[j] = Store<S>::raw(fin + (j * V + c + off));
            continue;
        }
        const bool cx = wx && ((ex_(j) > 0 && lox) || (ex_(j) < 0 && hix));
        const bool cy = wy && ((ey_(j) > 0 && loy) || (ey_(j) < 0 && hiy));
        const bool cz = wz && ((ez_(j) > 0 && loz) || (ez_(j) < 0 && hiz));
        // Source slot: the neighbour's j, or for a wall crossing this cell's
        // bi.  Only the index differs between the lanes, so a warp holding a
        // wall lane still issues one load per direction.
        // Written as selects (no branch), so the 15 loads stay one block.
        const int ix = P.face[ex_(j) > 0 ? 0 : 1].ubc == U_SPECULAR ? spec_(0, j) : opp_(j);
        const int iy = P.face[ey_(j) > 0 ? 2 : 3].ubc == U_SPECULAR ? spec_(1, j) : opp_(j);
        const int iz = P.face[ez_(j) > 0 ? 4 : 5].ubc == U_SPECULAR ? spec_(2, j) : opp_(j);
        int bi = cx ? ix : -1;
        bi = (cy && iy >= bi) ? iy : bi;
        bi = (cz && iz >= bi) ? iz : bi;
        const I src = (cx || cy || cz) ? (I)bi * V + c : j * V + c + off;
        raw[j] = Store<S>::raw(fin + src);
    }
#pragma unroll
    for (int j = 0; j < 15; ++j) f[j] = Store<S>::widen(raw[j]);
    if constexpr (WALLS) {
        if (P.moving_any) {
#pragma unroll
            for (int j = 0; j < 15; ++j) {
                const bool cx = wx && ((ex_(j) > 0 && lox) || (ex_(j) < 0 && hix));
                const bool cy = wy && ((ey_(j) > 0 && loy) || (ey_(j) < 0 && hiy));
                const bool cz = wz && ((ez_(j) > 0 && loz) || (ez_(j) < 0 && hiz));
                if (!(cx || cy || cz)) continue;
                int bf;
                wall_source(P, j, cx, cy, cz, &bf);
                if (P.face[bf].ubc == U_MOVING) {
                    const R dot = R(ex_(j)) * K.uw[bf][0] + R(ey_(j)) * K.uw[bf][1] + R(ez_(j)) * K.uw[bf][2];
                    f[j] = f[j] + R(6.0) * rho_prev * w_<R>(j) * dot;
                }
            }
        }
    }
}

// BGK relaxation with Guo forcing for the FP32 instantiations, by opposite
// pairs (j, opp(j)), e_opp = -e_j: with ue = e_j.u and eF = e_j.F, the
// equilibrium and forcing terms split into a part even in (ue, eF) and an
// odd part that flips sign, so one evaluation serves both directions:
//   f_j   <- om f_j   + G + H,   f_opp <- om f_opp + G - H,
//   G = omp w (s + rho (4.5 ue^2 - 1.5 u^2)) + DT omf w (9 ue eF - 3 u.F)
//       (DEV; plain storage has w rho (1 + ...) in place of w (s + rho ...)),
//   H = omp w rho 3 ue + DT omf w 3 eF.
// The same values as the direction-by-direction form (which the FP64 path
// keeps for bitwise parity) up to rounding.
template <class R, bool DEV>
__device__ __forceinline__ void relax_pairs(R om, R omp, R omf, R DT, R s, R rho, R ux, R uy, R uz, R Fx, R Fy,
                                            R Fz, R uF, R u2, R f[15]) {
    const R t = R(1.5) * u2, m3uF = R(-3.0) * uF, r3 = R(3.0) * rho;
    {
        const R w = w_<R>(0);
        const R feq = DEV ? w * (s - rho * t) : w * rho * (R(1.0) - t);
        f[0] = om * f[0] + (omp * feq + DT * omf * w * m3uF);
    }
#pragma unroll
    for (int j = 1; j < 15; ++j) {
        if (opp_(j) < j) continue;
        const int o = opp_(j);
        const R w = w_<R>(j);
        const R cw = omp * w, fw = DT * omf * w;
        const R ue = edot<R>(ex_(j), ey_(j), ez_(j), ux, uy, uz);
        const R eF = edot<R>(ex_(j), ey_(j), ez_(j), Fx, Fy, Fz);
        const R A = R(4.5) * ue * ue - t;
        const R even = DEV ? s + rho * A : rho * (R(1.0) + A);
        const R G = cw * even + fw * (R(9.0) * ue * eF + m3uF);
        const R H = cw * (r3 * ue) + fw * (R(3.0) * eF);
        const R fj = f[j], fo = f[o];
        f[j] = om * fj + (G + H);
        f[o] = om * fo + (G - H);
    }
}

// Moments, equilibrium, Guo forcing and BGK relaxation of one cell
// (src/physics_helpers.h:69-129); f is overwritten with f*.
template <class R, bool DEV>
__device__ __forceinline__ void collide(const Phys<R>& K, R f[15], R Fx, R Fy, R Fz, R& rho, R& ux,
                                        R& uy, R& uz) {
    const R DT = K.DT;
    R s, jx = R(0), jy = R(0), jz = R(0);
    if constexpr (sizeof(R) == 4) {
        // FP32: by opposite pairs, s = f0 + sum (f_j + f_opp) and
        // j = sum e_j (f_j - f_opp) -- shorter dependency chains.
        s = f[0];
        bool hx = false, hy = false, hz = false;
#pragma unroll
        for (int j = 1; j < 15; ++j) {
            if (opp_(j) < j) continue;
            const R p = f[j] + f[opp_(j)], m = f[j] - f[opp_(j)];
            s = s + p;
            if (ex_(j)) { const R t = sgn_term(ex_(j), m); jx = hx ? jx + t : t; hx = true; }
            if (ey_(j)) { const R t = sgn_term(ey_(j), m); jy = hy ? jy + t : t; hy = true; }
            if (ez_(j)) { const R t = sgn_term(ez_(j), m); jz = hz ? jz + t : t; hz = true; }
        }
    } else {  // the reference's summation order, for bitwise FP64 parity
        s = f[0];
#pragma unroll
        for (int j = 1; j < 15; ++j) s = s + f[j];
        bool hx = false, hy = false, hz = false;
#pragma unroll
        for (int j = 0; j < 15; ++j) {
            if (ex_(j)) { const R t = sgn_term(ex_(j), f[j]); jx = hx ? jx + t : t; hx = true; }
            if (ey_(j)) { const R t = sgn_term(ey_(j), f[j]); jy = hy ? jy + t : t; hy = true; }
            if (ez_(j)) { const R t = sgn_term(ez_(j), f[j]); jz = hz ? jz + t : t; hz = true; }
        }
    }
    const R rho0 = K.kDensity;
    rho = DEV ? rho0 + s : s;  // DEV: s is the density deviation
    if constexpr (sizeof(R) == 8) {  // the reference's divisions, for bitwise FP64 parity
        ux = (jx + R(0.5) * Fx * DT) / rho;
        uy = (jy + R(0.5) * Fy * DT) / rho;
        uz = (jz + R(0.5) * Fz * DT) / rho;
    } else {
        const R inv = R(1) / rho;
        ux = (jx + R(0.5) * Fx * DT) * inv;
        uy = (jy + R(0.5) * Fy * DT) * inv;
        uz = (jz + R(0.5) * Fz * DT) * inv;
    }
    const R uF = ux * Fx + uy * Fy + uz * Fz;
    const R u2 = ux * ux + uy * uy + uz * uz;
    const R om = K.omega, omp = K.omega_prime, omf = K.omega_forcing;
    if constexpr (sizeof(R) == 4) {
        relax_pairs<R, DEV>(om, omp, omf, DT, s, rho, ux, uy, uz, Fx, Fy, Fz, uF, u2, f);
    } else {
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
}

// Pre-collision populations of cell c: read in place on the first step after
// an upload, gathered from the neighbours' f* otherwise.
template <class R, class S, bool WALLS = true, class I = int64_t>
__device__ __forceinline__ void load_pre(const SimParams& P, const Phys<R>& K, bool first,
                                         const S* __restrict__ fin, I c, CellPos q, R rho_prev, R f[15]) {
    if (first) {
#pragma unroll
        for (int j = 0; j < 15; ++j) f[j] = Store<S>::ld(fin + (j * (I)P.V + c));
    } else {
        gather<R, S, WALLS, I>(P, K, fin, c, q, rho_prev, f);
    }
}

// Resident blocks per SM the LBM kernel's registers are held to (measured
// on B200: the walled form keeps its 15 loads in flight within 5 blocks per
// SM, 2 for FP64; the periodic form's natural budgets are 5 / 6 / 3 blocks for
// FP32 / FP16 storage / FP64).
template <class R, class S, bool WALLS>
constexpr int lbm_min_blocks() {
    return sizeof(R) == 8 ? (WALLS ? 2 : 3) : (sizeof(S) == 2 && !WALLS ? 6 : 5);
}

// One LBM step.  first: fin holds pre-collision populations (just uploaded).
// WALLS = false for boxes whose velocity axes are all periodic; I = int when
// 15 V < 2^31 (32-bit index arithmetic), else int64_t.
template <class R, class S, bool DEV, bool WALLS, class I>
__global__ void __launch_bounds__(256, lbm_min_blocks<R, S, WALLS>()) lbm_kernel(const __grid_constant__ SimParams P, FastDiv dnx, FastDiv dnxy, int first,
                                                  const S* __restrict__ fin, S* __restrict__ fout,
                                                  const R* __restrict__ F, R* __restrict__ rho_buf,
                                                  R* __restrict__ uout, int write_rho_all) {
    const I c = (I)blockIdx.x * (I)blockDim.x + (I)threadIdx.x;
    if (c >= (I)P.V) return;
    const I V = (I)P.V;
    const Phys<R>& K = phys_ref<R>(P);
    CellPos q;
    q.z = (int)fdiv((uint32_t)c, dnxy);
    const uint32_t r = (uint32_t)((int64_t)c - (int64_t)q.z * P.nxy);
    q.y = (int)fdiv(r, dnx);
    q.x = (int)(r - (uint32_t)q.y * (uint32_t)P.nx);
    const bool mv = WALLS && P.moving_any && touches_moving(P, q.x, q.y, q.z);
    R f[15];
    load_pre<R, S, WALLS, I>(P, K, first != 0, fin, c, q, (mv && !first) ? rho_buf[c] : R(0), f);
    R rho, ux, uy, uz;
    collide<R, DEV>(K, f, F[c], F[V + c], F[2 * V + c], rho, ux, uy, uz);
#pragma unroll
    for (int j = 0; j < 15; ++j) Store<S>::st(fout + j * V + c, f[j]);
    uout[c] = ux;
    uout[V + c] = uy;
    uout[2 * V + c] = uz;
    if (write_rho_all || mv) rho_buf[c] = rho;
}

// ---- in-place streaming (AA pattern), one population buffer ---------------
//
// The buffer alternates between two layouts:
//   PRE  : F[i][c] = pre-collision f_i(c) (what an upload leaves, and what
//          the reference stores);
//   SWAP : F[opp(i)][c] = post-collision f*_i(c).
// Even step (PRE -> SWAP): each cell reads its own 15 slots, collides and
// writes f*_i into its own slot opp(i).
// Odd step (SWAP -> PRE): each cell gathers f_j(c) = f*_j(c - e_j) from slot
// opp(j) of cell c - e_j (periodic axes wrap), or, when c - e_j lies beyond
// a wall, from its own slot opp(bi) holding f*_bi(c) (bi: the source the
// reference's wall rules leave in slot j, as in gather() above; a moving
// wall adds 6 rho w_j (e_j . U) with rho of the even step); it collides and
// scatters: f*_k to slot k of cell c + e_k, or, when c + e_k lies beyond a
// wall, f*_bi(opp k) (+ the moving-wall term with this step's rho) to its own
// slot opp(k) -- the pre-collision value the next even step reads there.
// Every slot is read and written by one thread only (the slot (k, x) of an
// odd step by cell x - e_k; a wall cell's own wall slots by itself), so one
// buffer serves both steps; the gathered values and the collision are those
// of the two-buffer kernel, bit for bit.

// Source of slot j of a wall cell: per crossed axis A the candidate opp(j)
// (no-slip / moving) or spec_A(j) (specular), the largest winning.  Also
// returns slot = opp(bi), where a SWAP-layout buffer holds f*_bi of the cell
// (chosen among compile-time candidates, so no table is indexed at run time).
__device__ __forceinline__ int wall_bi(const SimParams& P, int j, bool cx, bool cy, bool cz, int& slot) {
    const bool sx = P.face[ex_(j) > 0 ? 0 : 1].ubc == U_SPECULAR;
    const bool sy = P.face[ey_(j) > 0 ? 2 : 3].ubc == U_SPECULAR;
    const bool sz = P.face[ez_(j) > 0 ? 4 : 5].ubc == U_SPECULAR;
    const int ix = sx ? spec_(0, j) : opp_(j), iy = sy ? spec_(1, j) : opp_(j), iz = sz ? spec_(2, j) : opp_(j);
    const int tx = sx ? opp_(spec_(0, j)) : j, ty = sy ? opp_(spec_(1, j)) : j, tz = sz ? opp_(spec_(2, j)) : j;
    int bi = cx ? ix : -1;
    slot = cx ? tx : 0;
    if (cy && iy >= bi) { bi = iy; slot = ty; }
    if (cz && iz >= bi) { bi = iz; slot = tz; }
    return bi;
}

// Adds the moving-wall term of slot j of a wall cell to v, as gather() does
// (same expression, so the FP32 contraction is the same).
template <class R>
__device__ __forceinline__ void add_moving_term(const SimParams& P, const Phys<R>& K, int j, bool cx, bool cy,
                                                bool cz, R rho, R& v) {
    int bf;
    wall_source(P, j, cx, cy, cz, &bf);
    if (P.face[bf].ubc == U_MOVING) {
        const R dot = R(ex_(j)) * K.uw[bf][0] + R(ey_(j)) * K.uw[bf][1] + R(ez_(j)) * K.uw[bf][2];
        v = v + R(6.0) * rho * w_<R>(j) * dot;
    }
}

// Cell offsets of c + e (e = +1 / -1) along each axis, periodic wrap folded
// in, and whether the cell is on the low / high face of each axis.
template <class I>
struct AxisOff {
    I xm, xp, ym, yp, zm, zp;
    bool lox, hix, loy, hiy, loz, hiz;
};
template <class I>
__device__ __forceinline__ AxisOff<I> axis_off(const SimParams& P, CellPos q) {
    AxisOff<I> o;
    const int nx = P.nx, ny = P.ny, nz = P.nz;
    const I nxy = (I)P.nxy;
    o.lox = q.x == 0; o.hix = q.x == nx - 1; o.loy = q.y == 0; o.hiy = q.y == ny - 1;
    o.loz = q.z == 0; o.hiz = q.z == nz - 1;
    o.xm = o.lox ? (I)(nx - 1) : (I)-1;
    o.xp = o.hix ? (I)(1 - nx) : (I)1;
    o.ym = o.loy ? (I)(ny - 1) * nx : -(I)nx;
    o.yp = o.hiy ? -(I)(ny - 1) * nx : (I)nx;
    o.zm = o.loz ? (I)(nz - 1) * nxy : -nxy;
    o.zp = o.hiz ? -(I)(nz - 1) * nxy : nxy;
    return o;
}
// offset of c - e_j (source of a gather)
template <class I>
__device__ __forceinline__ I src_off(const AxisOff<I>& o, int j) {
    return (ex_(j) > 0 ? o.xm : ex_(j) < 0 ? o.xp : (I)0) + (ey_(j) > 0 ? o.ym : ey_(j) < 0 ? o.yp : (I)0) +
           (ez_(j) > 0 ? o.zm : ez_(j) < 0 ? o.zp : (I)0);
}
// does c - e_j lie beyond a wall, per axis.  WM: the axes that may have
// walls (bit 0 x, 1 y, 2 z), a compile-time superset of the box's walled
// axes, so directions and axes that cannot cross cost nothing.
template <int WM, class I>
__device__ __forceinline__ void crossing(const SimParams& P, const AxisOff<I>& o, int j, bool& cx, bool& cy,
                                         bool& cz) {
    cx = (WM & 1) && ex_(j) != 0 && !P.uper[0] && ((ex_(j) > 0 && o.lox) || (ex_(j) < 0 && o.hix));
    cy = (WM & 2) && ey_(j) != 0 && !P.uper[2] && ((ey_(j) > 0 && o.loy) || (ey_(j) < 0 && o.hiy));
    cz = (WM & 4) && ez_(j) != 0 && !P.uper[4] && ((ez_(j) > 0 && o.loz) || (ez_(j) < 0 && o.hiz));
}

template <class R, class S, bool DEV, int WM, class I>
__global__ void __launch_bounds__(256, lbm_min_blocks<R, S, WM != 0>())
    lbm_aa_even_kernel(const __grid_constant__ SimParams P, FastDiv dnx, FastDiv dnxy, S* F, const R* __restrict__ Fb,
                       R* __restrict__ rho_buf, R* __restrict__ uout, int write_rho_all) {
    const I c = (I)P.c0 + (I)blockIdx.x * (I)blockDim.x + (I)threadIdx.x;
    if (c >= (I)P.c1) return;
    const I V = (I)P.V;
    const Phys<R>& K = phys_ref<R>(P);
    S raw[15];
#pragma unroll
    for (int j = 0; j < 15; ++j) raw[j] = F[j * V + c];
    R f[15];
#pragma unroll
    for (int j = 0; j < 15; ++j) f[j] = Store<S>::widen(raw[j]);
    R rho, ux, uy, uz;
    collide<R, DEV>(K, f, Fb[c], Fb[V + c], Fb[2 * V + c], rho, ux, uy, uz);
#pragma unroll
    for (int j = 0; j < 15; ++j) Store<S>::st(F + opp_(j) * V + c, f[j]);
    uout[c] = ux;
    uout[V + c] = uy;
    uout[2 * V + c] = uz;
    bool mv = false;
    if (WM != 0 && P.moving_any && !write_rho_all) {
        CellPos q;
        q.z = (int)fdiv((uint32_t)c, dnxy);
        const uint32_t r = (uint32_t)((int64_t)c - (int64_t)q.z * P.nxy);
        q.y = (int)fdiv(r, dnx);
        q.x = (int)(r - (uint32_t)q.y * (uint32_t)P.nx);
        mv = touches_moving(P, q.x, q.y, q.z);
    }
    if (write_rho_all || mv) rho_buf[c] = rho;
}

template <class R, class S, bool DEV, int WM, class I>
__global__ void __launch_bounds__(256, lbm_min_blocks<R, S, WM != 0>())
    lbm_aa_odd_kernel(const __grid_constant__ SimParams P, FastDiv dnx, FastDiv dnxy, S* F, const R* __restrict__ Fb,
                      R* __restrict__ rho_buf, R* __restrict__ uout, int write_rho_all) {
    const I c = (I)P.c0 + (I)blockIdx.x * (I)blockDim.x + (I)threadIdx.x;
    if (c >= (I)P.c1) return;
    const I V = (I)P.V;
    const Phys<R>& K = phys_ref<R>(P);
    CellPos q;
    q.z = (int)fdiv((uint32_t)c, dnxy);
    const uint32_t r = (uint32_t)((int64_t)c - (int64_t)q.z * P.nxy);
    q.y = (int)fdiv(r, dnx);
    q.x = (int)(r - (uint32_t)q.y * (uint32_t)P.nx);
    const AxisOff<I> o = axis_off<I>(P, q);
    constexpr bool WALLS = WM != 0;
    const bool mv = WALLS && P.moving_any && touches_moving(P, q.x, q.y, q.z);
    const R rho_prev = mv ? rho_buf[c] : R(0);
    // gather: all 15 loads issued before the first widening
    S raw[15];
#pragma unroll
    for (int j = 0; j < 15; ++j) {
        if constexpr (!WALLS) {
            raw[j] = F[opp_(j) * V + c + src_off<I>(o, j)];
        } else {
            bool cx, cy, cz;
            crossing<WM, I>(P, o, j, cx, cy, cz);
            int slot;
            wall_bi(P, j, cx, cy, cz, slot);
            const I src = (cx || cy || cz) ? (I)slot * V + c : (I)opp_(j) * V + c + src_off<I>(o, j);
            raw[j] = F[src];
        }
    }
    R f[15];
#pragma unroll
    for (int j = 0; j < 15; ++j) f[j] = Store<S>::widen(raw[j]);
    if constexpr (WALLS) {
        if (mv) {
#pragma unroll
            for (int j = 0; j < 15; ++j) {
                bool cx, cy, cz;
                crossing<WM, I>(P, o, j, cx, cy, cz);
                if (!(cx || cy || cz)) continue;
                add_moving_term<R>(P, K, j, cx, cy, cz, rho_prev, f[j]);
            }
        }
    }
    R rho, ux, uy, uz;
    collide<R, DEV>(K, f, Fb[c], Fb[V + c], Fb[2 * V + c], rho, ux, uy, uz);
    // scatter
#pragma unroll
    for (int k = 0; k < 15; ++k) {
        if constexpr (!WALLS) {
            Store<S>::st(F + k * V + c + src_off<I>(o, opp_(k)), f[k]);  // c - e_opp(k) = c + e_k
        } else {
            // c + e_k beyond a wall <=> c - e_j beyond it for j = opp(k).  The
            // wall value is chosen among the compile-time candidates of
            // wall_bi (the largest source index wins), and the store address
            // and value by selects, so wall lanes do not split the warp.
            const int j = opp_(k);
            bool cx, cy, cz;
            crossing<WM, I>(P, o, j, cx, cy, cz);
            const bool sx = P.face[ex_(j) > 0 ? 0 : 1].ubc == U_SPECULAR;
            const bool sy = P.face[ey_(j) > 0 ? 2 : 3].ubc == U_SPECULAR;
            const bool sz = P.face[ez_(j) > 0 ? 4 : 5].ubc == U_SPECULAR;
            const int ix = sx ? spec_(0, j) : opp_(j), iy = sy ? spec_(1, j) : opp_(j), iz = sz ? spec_(2, j) : opp_(j);
            const R fx = sx ? f[spec_(0, j)] : f[opp_(j)], fy = sy ? f[spec_(1, j)] : f[opp_(j)];
            const R fz = sz ? f[spec_(2, j)] : f[opp_(j)];
            int bi = cx ? ix : -1;
            R v = cx ? fx : f[k];
            if (cy && iy >= bi) { bi = iy; v = fy; }
            if (cz && iz >= bi) { v = fz; }
            const bool cross = cx || cy || cz;
            if (mv && cross) add_moving_term<R>(P, K, j, cx, cy, cz, rho, v);
            Store<S>::st(F + (cross ? (I)j * V + c : (I)k * V + c + src_off<I>(o, j)), v);
        }
    }
    uout[c] = ux;
    uout[V + c] = uy;
    uout[2 * V + c] = uz;
    if (write_rho_all || mv) rho_buf[c] = rho;
}

// ---- in-place streaming, FP16 storage, two cells per thread ---------------
//
// The one-cell FP16 kernels above are bound by instruction issue (issue
// active 60-76%, DRAM 51-56% in a profile of a periodic 512x512x64 box).
// These forms update the cells c and c + 1 (c even; nx even, so c, V, c0 and
// c1 are even and each pair of slots (c, c + 1) is one aligned 4-byte word):
// the cell position, wrap offsets and slot addresses are computed once for
// both cells, and a population of both cells moves with one __half2 access
// wherever their slots are adjacent -- all 15 loads and stores of the even
// step, and the 5 directions without an x component in the odd step (the
// other 10 go to x - 1 or x + 1, whose pair straddles a word, and stay 2-byte
// accesses).  Velocity axes all periodic (no wall rules).  Each cell's
// arithmetic is that of the one-cell kernels (same collide, same
// conversions), so the result is the same bit for bit; the slots a thread
// reads and writes are the union of its two cells' slots, so the AA pattern
// stays race-free.  Plain loads on F: this kernel writes it.  (Device code
// only: host C++ checks of this header skip it.)
#if defined(__CUDACC__)
template <bool DEV, class I>
__global__ void __launch_bounds__(256, 4)
    lbm_aa_even_h2_kernel(const __grid_constant__ SimParams P, __half* F, const float* __restrict__ Fb,
                          float* __restrict__ rho_buf, float* __restrict__ uout, int write_rho_all) {
    const I c = (I)P.c0 + 2 * ((I)blockIdx.x * (I)blockDim.x + (I)threadIdx.x);
    if (c >= (I)P.c1) return;
    const I V = (I)P.V;
    const Phys<float>& K = phys_ref<float>(P);
    __half2 w[15];
#pragma unroll
    for (int j = 0; j < 15; ++j) w[j] = *reinterpret_cast<const __half2*>(F + j * V + c);
    float f[15];
    float rho, ux, uy, uz;
    // cell c; its post-collision values replace the low halves
#pragma unroll
    for (int j = 0; j < 15; ++j) f[j] = __low2float(w[j]);
    collide<float, DEV>(K, f, __ldg(Fb + c), __ldg(Fb + V + c), __ldg(Fb + 2 * V + c), rho, ux, uy, uz);
#pragma unroll
    for (int j = 0; j < 15; ++j) w[j] = __halves2half2(__float2half_rn(f[j]), __high2half(w[j]));
    uout[c] = ux;
    uout[V + c] = uy;
    uout[2 * V + c] = uz;
    if (write_rho_all) rho_buf[c] = rho;
    // cell c + 1
    const I c1 = c + 1;
#pragma unroll
    for (int j = 0; j < 15; ++j) f[j] = __high2float(w[j]);
    collide<float, DEV>(K, f, __ldg(Fb + c1), __ldg(Fb + V + c1), __ldg(Fb + 2 * V + c1), rho, ux, uy, uz);
    // V through an empty asm: the 15 store addresses are formed here rather
    // than kept live from the loads across both collisions (64 registers and
    // 4 blocks per SM instead of 80 and 3)
    I Vs = V;
    if constexpr (sizeof(I) == 4) asm volatile("" : "+r"(Vs));
    else asm volatile("" : "+l"(Vs));
#pragma unroll
    for (int j = 0; j < 15; ++j) {
        const __half2 v = __halves2half2(__low2half(w[j]), __float2half_rn(f[j]));
        *reinterpret_cast<__half2*>(F + opp_(j) * Vs + c) = v;  // f*_j into slot opp(j)
    }
    uout[c1] = ux;
    uout[V + c1] = uy;
    uout[2 * V + c1] = uz;
    if (write_rho_all) rho_buf[c1] = rho;
}

template <bool DEV, class I>
__global__ void __launch_bounds__(256, 3)
    lbm_aa_odd_h2_kernel(const __grid_constant__ SimParams P, FastDiv dnx, FastDiv dnxy, __half* F,
                         const float* __restrict__ Fb, float* __restrict__ rho_buf, float* __restrict__ uout,
                         int write_rho_all) {
    const I c = (I)P.c0 + 2 * ((I)blockIdx.x * (I)blockDim.x + (I)threadIdx.x);
    if (c >= (I)P.c1) return;
    const I V = (I)P.V;
    const Phys<float>& K = phys_ref<float>(P);
    CellPos q;
    q.z = (int)fdiv((uint32_t)c, dnxy);
    const uint32_t r = (uint32_t)((int64_t)c - (int64_t)q.z * P.nxy);
    q.y = (int)fdiv(r, dnx);
    q.x = (int)(r - (uint32_t)q.y * (uint32_t)P.nx);
    const AxisOff<I> o0 = axis_off<I>(P, q);  // cell c (x even)
    CellPos q1 = q;
    q1.x += 1;
    const AxisOff<I> o1 = axis_off<I>(P, q1);  // cell c + 1: only the x offsets differ
    // gather: every load of both cells issued before the first widening;
    // directions without an x component load both cells as one word, the
    // others load two halves, packed into one word once all are in flight
    __half2 w[15];
    __half a[15], b[15];
#pragma unroll
    for (int j = 0; j < 15; ++j) {
        if (ex_(j) == 0) {
            w[j] = *reinterpret_cast<const __half2*>(F + opp_(j) * V + c + src_off<I>(o0, j));
        } else {
            a[j] = F[opp_(j) * V + c + src_off<I>(o0, j)];
            b[j] = F[opp_(j) * V + c + 1 + src_off<I>(o1, j)];
        }
    }
#pragma unroll
    for (int j = 0; j < 15; ++j)
        if (ex_(j) != 0) w[j] = __halves2half2(a[j], b[j]);
    float f[15];
    float rho, ux, uy, uz;
    // cell c; the directions without an x component keep its value in the
    // low half until cell c + 1's joins it
#pragma unroll
    for (int j = 0; j < 15; ++j) f[j] = __low2float(w[j]);
    collide<float, DEV>(K, f, __ldg(Fb + c), __ldg(Fb + V + c), __ldg(Fb + 2 * V + c), rho, ux, uy, uz);
    // scatter: f*_k to slot k of c + e_k (= c - e_opp(k))
#pragma unroll
    for (int k = 0; k < 15; ++k) {
        if (ex_(k) == 0) w[k] = __halves2half2(__float2half_rn(f[k]), __high2half(w[k]));
        else Store<__half>::st(F + k * V + c + src_off<I>(o0, opp_(k)), f[k]);
    }
    uout[c] = ux;
    uout[V + c] = uy;
    uout[2 * V + c] = uz;
    if (write_rho_all) rho_buf[c] = rho;
    // cell c + 1
    const I c1 = c + 1;
#pragma unroll
    for (int j = 0; j < 15; ++j) f[j] = __high2float(w[j]);
    collide<float, DEV>(K, f, __ldg(Fb + c1), __ldg(Fb + V + c1), __ldg(Fb + 2 * V + c1), rho, ux, uy, uz);
#pragma unroll
    for (int k = 0; k < 15; ++k) {
        if (ex_(k) == 0) {
            const __half2 v = __halves2half2(__low2half(w[k]), __float2half_rn(f[k]));
            *reinterpret_cast<__half2*>(F + k * V + c + src_off<I>(o0, opp_(k))) = v;
        } else {
            Store<__half>::st(F + k * V + c1 + src_off<I>(o1, opp_(k)), f[k]);
        }
    }
    uout[c1] = ux;
    uout[V + c1] = uy;
    uout[2 * V + c1] = uz;
    if (write_rho_all) rho_buf[c1] = rho;
}
#endif  // __CUDACC__

// Pre-collision populations of direction j from a SWAP-layout buffer (for a
// download of f): the odd step's gather of one direction.
template <class R, class S>
__device__ __forceinline__ R aa_pre_population(const SimParams& P, const Phys<R>& K, const S* F, int64_t c,
                                               CellPos q, int j, const R* rho_buf) {
    const int64_t V = P.V;
    const AxisOff<int64_t> o = axis_off<int64_t>(P, q);
    bool cx, cy, cz;
    crossing<7, int64_t>(P, o, j, cx, cy, cz);
    if (!(cx || cy || cz)) return Store<S>::widen(F[opp_(j) * V + c + src_off<int64_t>(o, j)]);
    int slot;
    wall_bi(P, j, cx, cy, cz, slot);
    R v = Store<S>::widen(F[(int64_t)slot * V + c]);
    if (P.moving_any && touches_moving(P, q.x, q.y, q.z)) add_moving_term<R>(P, K, j, cx, cy, cz, rho_buf[c], v);
    return v;
}

// Download of direction dir from a SWAP-layout buffer, as float64 (the
// deviation offset w_dir rho0 added back).
template <class R, class S, bool DEV>
__global__ void __launch_bounds__(256) aa_pop_out_kernel(const __grid_constant__ SimParams P, FastDiv dnx,
                                                         FastDiv dnxy, const S* F, const R* __restrict__ rho_buf,
                                                         double* __restrict__ dst, int dir) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= P.V) return;
    CellPos q;
    q.z = (int)fdiv((uint32_t)c, dnxy);
    const uint32_t r = (uint32_t)(c - (int64_t)q.z * P.nxy);
    q.y = (int)fdiv(r, dnx);
    q.x = (int)(r - (uint32_t)q.y * (uint32_t)P.nx);
    const R v = aa_pre_population<R, S>(P, phys_ref<R>(P), F, c, q, dir, rho_buf);
    dst[c] = (double)v + (DEV ? w_<double>(dir) * P.kDensity : 0.0);
}

// Merge of the populations a neighbouring z-slab scattered across face
// `face` (0: low, 1: high) in an odd in-place step into this slab's owned
// boundary plane (zlo or zhi - 1).  They arrive staged as 5 planes, the
// slots k crossing that face (e_z = +1 at the low face, -1 at the high face)
// in increasing order.  Slot k of cell c holds f*_k of the source c - e_k;
// where that source lies beyond an x or y wall, the neighbour has no thread
// for it and this cell's own wall rule wrote the slot in the same step, so
// the slot is kept (the reference's unpack skip rule,
// src/mpi/halo_exchange_lbm.h SkipUnpackXY).
template <class S>
__global__ void __launch_bounds__(256) halo_merge_kernel(const __grid_constant__ SimParams P, S* F,
                                                         const S* __restrict__ stage, int face) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= P.nxy) return;
    const int y = (int)(t / P.nx), x = (int)(t - (int64_t)y * P.nx);
    const int64_t c = (int64_t)(face == 0 ? P.zlo : P.zhi - 1) * P.nxy + t;
    const int ez = face == 0 ? 1 : -1;
    int n = 0;
#pragma unroll
    for (int k = 1; k < 15; ++k) {
        if (ez_(k) != ez) continue;
        const bool cx = ex_(k) != 0 && !P.uper[0] && ((ex_(k) > 0 && x == 0) || (ex_(k) < 0 && x == P.nx - 1));
        const bool cy = ey_(k) != 0 && !P.uper[2] && ((ey_(k) > 0 && y == 0) || (ey_(k) < 0 && y == P.ny - 1));
        if (!cx && !cy) F[k * P.V + c] = stage[n * P.nxy + t];
        ++n;
    }
}

// In-place exchange of the direction slots j and opp(j) of every cell:
// converts the post-collision populations between the two-buffer layout
// (F[i][c] = f*_i(c)) and the SWAP layout (F[opp(i)][c] = f*_i(c)).
template <class S>
__global__ void __launch_bounds__(256) swap_pairs_kernel(int64_t V, S* F) {
    const int64_t c = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= V) return;
#pragma unroll
    for (int j = 1; j < 15; ++j) {
        if (opp_(j) < j) continue;
        const S a = F[j * V + c], b = F[opp_(j) * V + c];
        F[j * V + c] = b;
        F[opp_(j) * V + c] = a;
    }
}

// Pre-collision populations from the stored post-collision ones (for a
// download of f): the gather alone.
template <class R, class S>
__global__ void __launch_bounds__(256) stream_only_kernel(const __grid_constant__ SimParams P, FastDiv dnx, FastDiv dnxy,
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
    gather<R, S>(P, phys_ref<R>(P), fin, c, q, mv ? rho_buf[c] : R(0), f);
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
    const R rho0 = phys_ref<R>(P).kDensity;
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
