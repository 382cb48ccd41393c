/*
 * lbman_oracle.c -- CPU restatement of lbman3d's per-timestep hot path.
 *
 * TEST INFRASTRUCTURE ONLY (the checker; see lbman_oracle.h).  Compile with
 * -ffp-contract=off so no multiply-add is fused: the association order of
 * every expression below follows the reference line by line, which is what
 * makes the FP64 results bitwise equal to the reference's own CPU path.
 */
#include "lbman_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* D3Q15 velocity set, weights and symmetry maps (src/lattice_stencil.h:42-76). */
static const int EX[15] = {0, 1, 0, -1, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
static const int EY[15] = {0, 0, 1, 0, -1, 0, 0, 1, 1, -1, -1, 1, 1, -1, -1};
static const int EZ[15] = {0, 0, 0, 0, 0, 1, -1, 1, 1, 1, 1, -1, -1, -1, -1};
static const double W[15] = {2.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9, 1.0 / 9,
                             1.0 / 72, 1.0 / 72, 1.0 / 72, 1.0 / 72, 1.0 / 72, 1.0 / 72,
                             1.0 / 72, 1.0 / 72};
static const int OPP[15] = {0, 3, 4, 1, 2, 6, 5, 13, 14, 11, 12, 9, 10, 7, 8};
static const int SPEC[3][15] = {
    {0, 3, 2, 1, 4, 5, 6, 8, 7, 10, 9, 12, 11, 14, 13},  /* X, src/lattice_stencil.h:76 */
    {0, 1, 4, 3, 2, 5, 6, 10, 9, 8, 7, 14, 13, 12, 11},  /* Y, :69 */
    {0, 1, 2, 3, 4, 6, 5, 11, 12, 13, 14, 7, 8, 9, 10},  /* Z, :62 */
};

struct orc_state {
    orc_params p;
    int64_t V;
    double omega, omega_prime, omega_forcing;
    double anchor[6][5];
    double *f, *f_new, *rho, *u[3], *F[3], *q[5], *q_new[5], *sig[5], *tau[3];
};

/* ---------------------------------------------------------------------- */
/* Parameters                                                              */

void orc_params_default(orc_params* p) {
    /* Defaults of src/params.h:14-112 with SimBC = SlitNoSlipConfig
     * (src/sim_config.h:37-48). */
    memset(p, 0, sizeof(*p));
    p->nx = 20; p->ny = 100; p->nz = 100;
    p->DT = 1.0; p->kDensity = 1.0; p->TAUF = 2.5 * 1.0;
    p->L = 0.06; p->A = 0; p->B = -0.3; p->C = 0.3;
    p->LAMBDA = 0.3; p->GAMMA = 0.34; p->ALPHA = 0.023; p->MU = 0.0;
    p->advection = ORC_CENTRED;
    for (int k = 0; k < 6; ++k) { p->face[k].qbc = ORC_Q_PERIODIC; p->face[k].ubc = ORC_U_PERIODIC; }
    p->face[0].qbc = p->face[1].qbc = ORC_Q_NEUMANN;
    p->face[0].ubc = p->face[1].ubc = ORC_U_NOSLIP;
}

/* src/boundary_handler.h:232-251 */
void orc_anchored_q(const orc_face* f, double out[5]) {
    if (f->qbc != ORC_Q_ANCHORING) { for (int k = 0; k < 5; ++k) out[k] = 0.0; return; }
    const double sin_sq_phi = 0.5 * (1.0 - cos(2.0 * f->phi));
    const double cos_sq_phi = 1.0 - sin_sq_phi;
    const double sin_phi_cos_phi = 0.5 * sin(2.0 * f->phi);
    const double sin_sq_th = 0.5 * (1.0 - cos(2.0 * f->theta));
    const double sin_th_cos_th = 0.5 * sin(2.0 * f->theta);
    const double S = f->s;
    out[0] = S * (cos_sq_phi * sin_sq_th - 1.0 / 3.0);
    out[1] = S * (sin_phi_cos_phi * sin_sq_th);
    out[2] = S * (cos(f->phi) * sin_th_cos_th);
    out[3] = S * (sin_sq_phi * sin_sq_th - 1.0 / 3.0);
    out[4] = S * (sin(f->phi) * sin_th_cos_th);
}

/* src/model.h:39-41 */
double orc_equilibrium_order(const orc_params* p) {
    return (-p->B + sqrt(p->B * p->B - 24.0 * p->A * p->C)) / (4.0 * p->C);
}

/* ---------------------------------------------------------------------- */
/* Index policies                                                          */

static inline int64_t cidx(const orc_params* p, int x, int y, int z) {
    return ((int64_t)z * p->ny + y) * p->nx + x;
}
static inline int wrapi(int i, int n) { return ((i % n) + n) % n; }
static inline int clampi(int t, int n) { return t < 0 ? 0 : (t >= n ? n - 1 : t); }

/* SafeFetchAxisOffset (src/boundary_handler.h:76-89) and QAxisOffset
 * (src/offsets.h:59-72): wrap on a periodic side, clamp otherwise. */
static inline int fetch_off(int lo_per, int hi_per, int i, int s, int n) {
    const int t = i + s;
    if (t < 0) return lo_per ? wrapi(t, n) : clampi(t, n);
    if (t >= n) return hi_per ? wrapi(t, n) : clampi(t, n);
    return t;
}

static inline int qper(const orc_params* p, int face) { return p->face[face].qbc == ORC_Q_PERIODIC; }
static inline int uper(const orc_params* p, int face) { return p->face[face].ubc == ORC_U_PERIODIC; }

/* ---------------------------------------------------------------------- */
/* Q gradient and Laplacian with wall ghosts (src/boundary_handler.h:253-320) */

typedef struct { double dx, dy, dz, lap, d2x, d2y, d2z; } qderivs;

static inline double q_ghost(const orc_state* s, int face, int comp, double qb) {
    if (s->p.face[face].qbc == ORC_Q_ANCHORING) return 2.0 * s->anchor[face][comp] - qb;
    return qb; /* Neumann clamp; a Periodic tag on a non-periodic Lo face lands here too */
}

/* QAxisGhostPair: the Lo face's tag decides whether ghosts apply at all. */
static inline void q_pair(const orc_state* s, int ax, int comp, int a, int n, double qm, double q0,
                          double qp, double* m, double* pl) {
    const int lo = 2 * ax, hi = 2 * ax + 1;
    if (s->p.face[lo].qbc == ORC_Q_PERIODIC) { *m = qm; *pl = qp; return; }
    *m = (a == 0) ? q_ghost(s, lo, comp, q0) : qm;
    *pl = (a == n - 1) ? q_ghost(s, hi, comp, q0) : qp;
}

static qderivs q_grad_lap(const orc_state* s, const double* q, int comp, int x, int y, int z) {
    const orc_params* p = &s->p;
    const int xm = fetch_off(qper(p, 0), qper(p, 1), x, -1, p->nx);
    const int xp = fetch_off(qper(p, 0), qper(p, 1), x, +1, p->nx);
    const int ym = fetch_off(qper(p, 2), qper(p, 3), y, -1, p->ny);
    const int yp = fetch_off(qper(p, 2), qper(p, 3), y, +1, p->ny);
    const int zm = fetch_off(qper(p, 4), qper(p, 5), z, -1, p->nz);
    const int zp = fetch_off(qper(p, 4), qper(p, 5), z, +1, p->nz);
    const double q0 = q[cidx(p, x, y, z)];
    double pxm, pxp, pym, pyp, pzm, pzp;
    q_pair(s, 0, comp, x, p->nx, q[cidx(p, xm, y, z)], q0, q[cidx(p, xp, y, z)], &pxm, &pxp);
    q_pair(s, 1, comp, y, p->ny, q[cidx(p, x, ym, z)], q0, q[cidx(p, x, yp, z)], &pym, &pyp);
    q_pair(s, 2, comp, z, p->nz, q[cidx(p, x, y, zm)], q0, q[cidx(p, x, y, zp)], &pzm, &pzp);
    qderivs d;
    d.dx = (pxp - pxm) / 2.0;
    d.dy = (pyp - pym) / 2.0;
    d.dz = (pzp - pzm) / 2.0;
    d.lap = (pxm + pxp + pym + pyp + pzm + pzp) - 6.0 * q0;
    d.d2x = (pxm + pxp) - 2.0 * q0;
    d.d2y = (pym + pyp) - 2.0 * q0;
    d.d2z = (pzm + pzp) - 2.0 * q0;
    return d;
}

/* ---------------------------------------------------------------------- */
/* Velocity gradient with wall ghosts (src/boundary_handler.h:112-209)     */

static inline double v_ghost(const orc_state* s, int face, int comp, double vb, int is_normal) {
    const orc_face* f = &s->p.face[face];
    const double wall = (f->ubc == ORC_U_MOVING) ? f->uw[comp] : 0.0;
    if (f->ubc == ORC_U_SPECULAR) return is_normal ? (2.0 * wall - vb) : vb;
    return 2.0 * wall - vb;
}

static inline double v_axis_grad(const orc_state* s, int ax, int comp, int a, int n, double vm,
                                 double vc, double vp, int is_normal) {
    const int lo = 2 * ax, hi = 2 * ax + 1;
    double m = vm, pl = vp;
    if (s->p.face[lo].ubc != ORC_U_PERIODIC) {
        m = (a == 0) ? v_ghost(s, lo, comp, vc, is_normal) : vm;
        pl = (a == n - 1) ? v_ghost(s, hi, comp, vc, is_normal) : vp;
    }
    return (pl - m) / 2.0;
}

typedef struct { double ux_x, ux_y, ux_z, uy_x, uy_y, uy_z, uz_x, uz_y; } gradu;

static gradu vel_grad(const orc_state* s, int x, int y, int z) {
    const orc_params* p = &s->p;
    const double *ux = s->u[0], *uy = s->u[1], *uz = s->u[2];
    const int xm = fetch_off(uper(p, 0), uper(p, 1), x, -1, p->nx);
    const int xp = fetch_off(uper(p, 0), uper(p, 1), x, +1, p->nx);
    const int ym = fetch_off(uper(p, 2), uper(p, 3), y, -1, p->ny);
    const int yp = fetch_off(uper(p, 2), uper(p, 3), y, +1, p->ny);
    const int zm = fetch_off(uper(p, 4), uper(p, 5), z, -1, p->nz);
    const int zp = fetch_off(uper(p, 4), uper(p, 5), z, +1, p->nz);
    const int64_t c = cidx(p, x, y, z);
    const double ux0 = ux[c], uy0 = uy[c], uz0 = uz[c];
    gradu g;
    g.ux_x = v_axis_grad(s, 0, 0, x, p->nx, ux[cidx(p, xm, y, z)], ux0, ux[cidx(p, xp, y, z)], 1);
    g.ux_y = v_axis_grad(s, 1, 0, y, p->ny, ux[cidx(p, x, ym, z)], ux0, ux[cidx(p, x, yp, z)], 0);
    g.ux_z = v_axis_grad(s, 2, 0, z, p->nz, ux[cidx(p, x, y, zm)], ux0, ux[cidx(p, x, y, zp)], 0);
    g.uy_x = v_axis_grad(s, 0, 1, x, p->nx, uy[cidx(p, xm, y, z)], uy0, uy[cidx(p, xp, y, z)], 0);
    g.uy_y = v_axis_grad(s, 1, 1, y, p->ny, uy[cidx(p, x, ym, z)], uy0, uy[cidx(p, x, yp, z)], 1);
    g.uy_z = v_axis_grad(s, 2, 1, z, p->nz, uy[cidx(p, x, y, zm)], uy0, uy[cidx(p, x, y, zp)], 0);
    g.uz_x = v_axis_grad(s, 0, 2, x, p->nx, uz[cidx(p, xm, y, z)], uz0, uz[cidx(p, xp, y, z)], 0);
    g.uz_y = v_axis_grad(s, 1, 2, y, p->ny, uz[cidx(p, x, ym, z)], uz0, uz[cidx(p, x, yp, z)], 0);
    return g;
}

/* ---------------------------------------------------------------------- */
/* Pointwise Beris-Edwards step (src/model.h:60-82 and 102-342)             */

static inline double adv_axis(int upwind, double u, double dQ, double d2Q) {
    if (upwind) {
        const double abs_u = u < 0.0 ? -u : u;
        return u * dQ - 0.5 * abs_u * d2Q;
    }
    return u * dQ;
}
static inline double adv_deriv(int upwind, const double u[3], const qderivs* d) {
    return adv_axis(upwind, u[0], d->dx, d->d2x) + adv_axis(upwind, u[1], d->dy, d->d2y) +
           adv_axis(upwind, u[2], d->dz, d->d2z);
}

static void pointwise_q(const orc_state* s, const double Q[5], const double u[3],
                        const qderivs d[5], const gradu* g, double qn[5], double sig[5],
                        double tau[3], double eric[3]) {
    const orc_params* p = &s->p;
    const double A = p->A, B = p->B, C = p->C, L = p->L, LAMBDA = p->LAMBDA, GAMMA = p->GAMMA,
                 DT = p->DT;
    const int up = p->advection == ORC_UPWIND;
    const double Qxx = Q[0], Qxy = Q[1], Qxz = Q[2], Qyy = Q[3], Qyz = Q[4];

    const double TrQ2 = 2.0 * (Qxx * Qxx + Qyy * Qyy + Qxx * Qyy + Qxy * Qxy + Qxz * Qxz + Qyz * Qyz);
    const double k13 = 1.0 / 3.0;
    const double Q2_xx = Qxx * Qxx + Qxy * Qxy + Qxz * Qxz - k13 * TrQ2;
    const double Q2_xy = Qxx * Qxy + Qxy * Qyy + Qxz * Qyz;
    const double Q2_xz = Qxy * Qyz - Qxz * Qyy;
    const double Q2_yy = Qxy * Qxy + Qyy * Qyy + Qyz * Qyz - k13 * TrQ2;
    const double Q2_yz = Qxy * Qxz - Qyz * Qxx;

    const double Exx = g->ux_x;
    const double Exy = 0.5 * (g->ux_y + g->uy_x);
    const double Exz = 0.5 * (g->ux_z + g->uz_x);
    const double Eyy = g->uy_y;
    const double Eyz = 0.5 * (g->uy_z + g->uz_y);
    const double Wxy = 0.5 * (g->ux_y - g->uy_x);
    const double Wxz = 0.5 * (g->ux_z - g->uz_x);
    const double Wyz = 0.5 * (g->uy_z - g->uz_y);

    const double Qxxx = d[0].dx, Qxxy = d[0].dy, Qxxz = d[0].dz;
    const double Qxyx = d[1].dx, Qxyy = d[1].dy, Qxyz = d[1].dz;
    const double Qxzx = d[2].dx, Qxzy = d[2].dy, Qxzz = d[2].dz;
    const double Qyyx = d[3].dx, Qyyy = d[3].dy, Qyyz = d[3].dz;
    const double Qyzx = d[4].dx, Qyzy = d[4].dy, Qyzz = d[4].dz;

    const double adv_xx = -adv_deriv(up, u, &d[0]);
    const double adv_xy = -adv_deriv(up, u, &d[1]);
    const double adv_xz = -adv_deriv(up, u, &d[2]);
    const double adv_yy = -adv_deriv(up, u, &d[3]);
    const double adv_yz = -adv_deriv(up, u, &d[4]);

    const double cor_xx = 2.0 * (Qxy * Wxy + Qxz * Wxz);
    const double cor_xy = -Qxx * Wxy + Qxz * Wyz + Qyy * Wxy + Qyz * Wxz;
    const double cor_xz = -2.0 * Qxx * Wxz - Qxy * Wyz - Qyy * Wxz + Qyz * Wxy;
    const double cor_yy = 2.0 * (-Qxy * Wxy + Qyz * Wyz);
    const double cor_yz = -Qxx * Wyz - Qxy * Wxz - Qxz * Wxy - 2.0 * Qyy * Wyz;

    const double k23 = 2.0 / 3.0;
    const double tr_QE = (2.0 * Exx + Eyy) * Qxx + (2.0 * Exy) * Qxy + (2.0 * Exz) * Qxz +
                         (Exx + 2.0 * Eyy) * Qyy + 2.0 * Eyz * Qyz;
    const double aln2_xx = 2.0 * (Exx * Qxx + Exy * Qxy + Exz * Qxz) - k23 * tr_QE;
    const double aln2_xy = Exy * Qxx + Eyy * Qxy + Eyz * Qxz + Qxy * Exx + Qyy * Exy + Qyz * Exz;
    const double aln2_xz =
        Exz * Qxx + Eyz * Qxy + (-Exx - Eyy) * Qxz + Qxz * Exx + Qyz * Exy + (-Qxx - Qyy) * Exz;
    const double aln2_yy = 2.0 * (Exy * Qxy + Eyy * Qyy + Eyz * Qyz) - k23 * tr_QE;
    const double aln2_yz =
        Exz * Qxy + Eyz * Qyy + (-Exx - Eyy) * Qyz + Qxz * Exy + Qyz * Eyy + (-Qxx - Qyy) * Eyz;
    const double aln3_xx = -2.0 * tr_QE * Qxx;
    const double aln3_xy = -2.0 * tr_QE * Qxy;
    const double aln3_xz = -2.0 * tr_QE * Qxz;
    const double aln3_yy = -2.0 * tr_QE * Qyy;
    const double aln3_yz = -2.0 * tr_QE * Qyz;

    const double ld = A + C * TrQ2;
    const double Hxx = L * d[0].lap - ld * Qxx - B * Q2_xx;
    const double Hxy = L * d[1].lap - ld * Qxy - B * Q2_xy;
    const double Hxz = L * d[2].lap - ld * Qxz - B * Q2_xz;
    const double Hyy = L * d[3].lap - ld * Qyy - B * Q2_yy;
    const double Hyz = L * d[4].lap - ld * Qyz - B * Q2_yz;

    eric[0] = -2.0 * (Hxx * Qxxx + Hxy * Qxyx + Hxz * Qxzx + Hyy * Qyyx + Hyz * Qyzx) - Hxx * Qyyx - Hyy * Qxxx;
    eric[1] = -2.0 * (Hxx * Qxxy + Hxy * Qxyy + Hxz * Qxzy + Hyy * Qyyy + Hyz * Qyzy) - Hxx * Qyyy - Hyy * Qxxy;
    eric[2] = -2.0 * (Hxx * Qxxz + Hxy * Qxyz + Hxz * Qxzz + Hyy * Qyyz + Hyz * Qyzz) - Hxx * Qyyz - Hyy * Qxxz;

    const double tr_QH = (2.0 * Hxx + Hyy) * Qxx + (2.0 * Hxy) * Qxy + (2.0 * Hxz) * Qxz +
                         (Hxx + 2.0 * Hyy) * Qyy + 2.0 * Hyz * Qyz;
    const double QHxx = 2.0 * (Hxx * Qxx + Hxy * Qxy + Hxz * Qxz) - k23 * tr_QH;
    const double QHxy = Hxy * Qxx + Hyy * Qxy + Hyz * Qxz + Qxy * Hxx + Qyy * Hxy + Qyz * Hxz;
    const double QHxz =
        Hxz * Qxx + Hyz * Qxy + (-Hxx - Hyy) * Qxz + Qxz * Hxx + Qyz * Hxy + (-Qxx - Qyy) * Hxz;
    const double QHyy = 2.0 * (Hxy * Qxy + Hyy * Qyy + Hyz * Qyz) - k23 * tr_QH;
    const double QHyz =
        Hxz * Qxy + Hyz * Qyy + (-Hxx - Hyy) * Qyz + Qxz * Hxy + Qyz * Hyy + (-Qxx - Qyy) * Hyz;

    tau[0] = (Hxy * Qxx + Hyy * Qxy + Hyz * Qxz) - (Qxy * Hxx + Qyy * Hxy + Qyz * Hxz);
    tau[1] = (Hxz * Qxx + Hyz * Qxy + (-Hxx - Hyy) * Qxz) - (Qxz * Hxx + Qyz * Hxy + (-Qxx - Qyy) * Hxz);
    tau[2] = (Hxz * Qxy + Hyz * Qyy + (-Hxx - Hyy) * Qyz) - (Qxz * Hxy + Qyz * Hyy + (-Qxx - Qyy) * Hyz);

    sig[0] = -k23 * LAMBDA * Hxx - LAMBDA * QHxx + 2.0 * LAMBDA * tr_QH * Qxx;
    sig[1] = -k23 * LAMBDA * Hxy - LAMBDA * QHxy + 2.0 * LAMBDA * tr_QH * Qxy;
    sig[2] = -k23 * LAMBDA * Hxz - LAMBDA * QHxz + 2.0 * LAMBDA * tr_QH * Qxz;
    sig[3] = -k23 * LAMBDA * Hyy - LAMBDA * QHyy + 2.0 * LAMBDA * tr_QH * Qyy;
    sig[4] = -k23 * LAMBDA * Hyz - LAMBDA * QHyz + 2.0 * LAMBDA * tr_QH * Qyz;

    qn[0] = Qxx + DT * (adv_xx + cor_xx + LAMBDA * (k23 * Exx + aln2_xx + aln3_xx) + GAMMA * Hxx);
    qn[1] = Qxy + DT * (adv_xy + cor_xy + LAMBDA * (k23 * Exy + aln2_xy + aln3_xy) + GAMMA * Hxy);
    qn[2] = Qxz + DT * (adv_xz + cor_xz + LAMBDA * (k23 * Exz + aln2_xz + aln3_xz) + GAMMA * Hxz);
    qn[3] = Qyy + DT * (adv_yy + cor_yy + LAMBDA * (k23 * Eyy + aln2_yy + aln3_yy) + GAMMA * Hyy);
    qn[4] = Qyz + DT * (adv_yz + cor_yz + LAMBDA * (k23 * Eyz + aln2_yz + aln3_yz) + GAMMA * Hyz);
}

/* ---------------------------------------------------------------------- */
/* State                                                                   */

orc_state* orc_new(const orc_params* p) {
    orc_state* s = (orc_state*)calloc(1, sizeof(orc_state));
    if (!s) return NULL;
    s->p = *p;
    s->V = (int64_t)p->nx * p->ny * p->nz;
    /* src/params.h:52-54 */
    s->omega = 1.0 - p->DT / p->TAUF;
    s->omega_prime = p->DT / p->TAUF;
    s->omega_forcing = 1.0 - p->DT / 2.0 / p->TAUF;
    for (int k = 0; k < 6; ++k) orc_anchored_q(&p->face[k], s->anchor[k]);
    const int64_t V = s->V;
    s->f = (double*)calloc((size_t)(15 * V), sizeof(double));
    s->f_new = (double*)calloc((size_t)(15 * V), sizeof(double));
    s->rho = (double*)calloc((size_t)V, sizeof(double));
    for (int k = 0; k < 3; ++k) {
        s->u[k] = (double*)calloc((size_t)V, sizeof(double));
        s->F[k] = (double*)calloc((size_t)V, sizeof(double));
        s->tau[k] = (double*)calloc((size_t)V, sizeof(double));
    }
    for (int k = 0; k < 5; ++k) {
        s->q[k] = (double*)calloc((size_t)V, sizeof(double));
        s->q_new[k] = (double*)calloc((size_t)V, sizeof(double));
        s->sig[k] = (double*)calloc((size_t)V, sizeof(double));
    }
    for (int64_t c = 0; c < V; ++c) s->rho[c] = p->kDensity;
    return s;
}

void orc_free(orc_state* s) {
    if (!s) return;
    free(s->f); free(s->f_new); free(s->rho);
    for (int k = 0; k < 3; ++k) { free(s->u[k]); free(s->F[k]); free(s->tau[k]); }
    for (int k = 0; k < 5; ++k) { free(s->q[k]); free(s->q_new[k]); free(s->sig[k]); }
    free(s);
}

/* LbmSolver::Initialize (src/lbm_solver.tpp:35-62) with Feq
 * (src/physics_helpers.h:69-71). */
static void lbm_init(orc_state* s) {
    const int64_t V = s->V;
    for (int64_t c = 0; c < V; ++c) {
        const double rhop = s->rho[c];
        const double ux = s->u[0][c], uy = s->u[1][c], uz = s->u[2][c];
        const double u2 = ux * ux + uy * uy + uz * uz;
        for (int i = 0; i < 15; ++i) {
            const double ue = ux * (double)EX[i] + uy * (double)EY[i] + uz * (double)EZ[i];
            s->f[i * V + c] = (W[i] * rhop * (1.0 + 3.0 * ue + 4.5 * ue * ue - 1.5 * u2));
        }
    }
}

void orc_set(orc_state* s, const double* rho, const double* u3, const double* q5,
             const double* f15, const double* force3) {
    const int64_t V = s->V;
    const size_t vb = (size_t)V * sizeof(double);
    if (rho) memcpy(s->rho, rho, vb);
    for (int k = 0; k < 3; ++k) {
        if (u3) memcpy(s->u[k], u3 + k * V, vb);
        if (force3) memcpy(s->F[k], force3 + k * V, vb); else memset(s->F[k], 0, vb);
    }
    if (q5) for (int k = 0; k < 5; ++k) memcpy(s->q[k], q5 + k * V, vb);
    if (f15) memcpy(s->f, f15, 15 * vb); else lbm_init(s);
}

void orc_get(const orc_state* s, double* rho, double* u3, double* q5, double* f15,
             double* force3, double* sigma5, double* tau3) {
    const int64_t V = s->V;
    const size_t vb = (size_t)V * sizeof(double);
    if (rho) memcpy(rho, s->rho, vb);
    for (int k = 0; k < 3; ++k) {
        if (u3) memcpy(u3 + k * V, s->u[k], vb);
        if (force3) memcpy(force3 + k * V, s->F[k], vb);
        if (tau3) memcpy(tau3 + k * V, s->tau[k], vb);
    }
    for (int k = 0; k < 5; ++k) {
        if (q5) memcpy(q5 + k * V, s->q[k], vb);
        if (sigma5) memcpy(sigma5 + k * V, s->sig[k], vb);
    }
    if (f15) memcpy(f15, s->f, 15 * vb);
}

/* ---------------------------------------------------------------------- */
/* QTensorSolver::StepAndSetupBodyForce (src/qtensor_solver.tpp:51-147)     */

static void q_step_setup(orc_state* s) {
    const orc_params* p = &s->p;
#pragma omp parallel for schedule(static)
    for (int z = 0; z < p->nz; ++z)
        for (int y = 0; y < p->ny; ++y)
            for (int x = 0; x < p->nx; ++x) {
                const int64_t c = cidx(p, x, y, z);
                double Q[5], u[3], qn[5], sg[5], ta[3], er[3];
                qderivs d[5];
                for (int k = 0; k < 5; ++k) Q[k] = s->q[k][c];
                for (int k = 0; k < 3; ++k) u[k] = s->u[k][c];
                for (int k = 0; k < 5; ++k) d[k] = q_grad_lap(s, s->q[k], k, x, y, z);
                const gradu g = vel_grad(s, x, y, z);
                pointwise_q(s, Q, u, d, &g, qn, sg, ta, er);
                for (int k = 0; k < 3; ++k) s->F[k][c] = er[k];
                for (int k = 0; k < 5; ++k) s->sig[k][c] = sg[k];
                for (int k = 0; k < 3; ++k) s->tau[k][c] = ta[k];
                for (int k = 0; k < 5; ++k) s->q_new[k][c] = qn[k];
            }
    for (int k = 0; k < 5; ++k) { double* t = s->q[k]; s->q[k] = s->q_new[k]; s->q_new[k] = t; }
}

/* QTensorSolver::SetActiveStressAndComputeBodyForce (src/qtensor_solver.tpp:155-217),
 * PassiveStressDivergence (src/boundary_handler.h:335-392) and
 * PointwiseSetActiveStressAndComputeBodyForce (src/model.h:344-361). */
static void body_force(orc_state* s) {
    const orc_params* p = &s->p;
    const double ALPHA = p->ALPHA, MU = p->MU;
#pragma omp parallel for schedule(static)
    for (int z = 0; z < p->nz; ++z)
        for (int y = 0; y < p->ny; ++y)
            for (int x = 0; x < p->nx; ++x) {
                const int64_t c = cidx(p, x, y, z);
                qderivs d[5];
                for (int k = 0; k < 5; ++k) d[k] = q_grad_lap(s, s->q[k], k, x, y, z);
                const int xm = fetch_off(qper(p, 0), qper(p, 1), x, -1, p->nx);
                const int xp = fetch_off(qper(p, 0), qper(p, 1), x, +1, p->nx);
                const int ym = fetch_off(qper(p, 2), qper(p, 3), y, -1, p->ny);
                const int yp = fetch_off(qper(p, 2), qper(p, 3), y, +1, p->ny);
                const int zm = fetch_off(qper(p, 4), qper(p, 5), z, -1, p->nz);
                const int zp = fetch_off(qper(p, 4), qper(p, 5), z, +1, p->nz);
                const int64_t cxm = cidx(p, xm, y, z), cxp = cidx(p, xp, y, z);
                const int64_t cym = cidx(p, x, ym, z), cyp = cidx(p, x, yp, z);
                const int64_t czm = cidx(p, x, y, zm), czp = cidx(p, x, y, zp);
                double* const* S = s->sig;
                double* const* T = s->tau;
                const double dx_Sxx = (S[0][cxp] - S[0][cxm]) / 2.0;
                const double dx_Sxy = (S[1][cxp] - S[1][cxm]) / 2.0;
                const double dx_Sxz = (S[2][cxp] - S[2][cxm]) / 2.0;
                const double dx_Txy = (T[0][cxp] - T[0][cxm]) / 2.0;
                const double dx_Txz = (T[1][cxp] - T[1][cxm]) / 2.0;
                const double dy_Sxy = (S[1][cyp] - S[1][cym]) / 2.0;
                const double dy_Syy = (S[3][cyp] - S[3][cym]) / 2.0;
                const double dy_Syz = (S[4][cyp] - S[4][cym]) / 2.0;
                const double dy_Txy = (T[0][cyp] - T[0][cym]) / 2.0;
                const double dy_Tyz = (T[2][cyp] - T[2][cym]) / 2.0;
                const double dz_Sxz = (S[2][czp] - S[2][czm]) / 2.0;
                const double dz_Syz = (S[4][czp] - S[4][czm]) / 2.0;
                const double dz_Txz = (T[1][czp] - T[1][czm]) / 2.0;
                const double dz_Tyz = (T[2][czp] - T[2][czm]) / 2.0;
                const double dz_Szz = -((S[0][czp] - S[0][czm]) / 2.0 + (S[3][czp] - S[3][czm]) / 2.0);
                const double pdx = dx_Sxx + (dy_Sxy + dy_Txy) + (dz_Sxz + dz_Txz);
                const double pdy = (dx_Sxy - dx_Txy) + dy_Syy + (dz_Syz + dz_Tyz);
                const double pdz = (dx_Sxz - dx_Txz) + (dy_Syz - dy_Tyz) + dz_Szz;
                const double fx = -ALPHA * (d[0].dx + d[1].dy + d[2].dz) + pdx - MU * s->u[0][c];
                const double fy = -ALPHA * (d[1].dx + d[3].dy + d[4].dz) + pdy - MU * s->u[1][c];
                const double fz = -ALPHA * (d[2].dx + d[4].dy - d[0].dz - d[3].dz) + pdz - MU * s->u[2][c];
                s->F[0][c] += fx;
                s->F[1][c] += fy;
                s->F[2][c] += fz;
            }
}

void orc_q_step(orc_state* s, int with_active) {
    q_step_setup(s);
    if (with_active) body_force(s);
}

/* ---------------------------------------------------------------------- */
/* LbmSolver::LatticeBoltzmannStep (src/lbm_solver.tpp:65-199), push form  */

/* StreamAxisOffset (src/boundary_handler.h:41-53): wrap on a periodic side,
 * raw (possibly out of domain) otherwise. */
static inline int stream_off(int lo_per, int hi_per, int i, int s, int n) {
    const int t = i + s;
    if (t < 0) return lo_per ? wrapi(t, n) : t;
    if (t >= n) return hi_per ? wrapi(t, n) : t;
    return t;
}

/* HandleBoundaryPoint (src/boundary_handler.h:403-426) */
static inline void handle_wall(const orc_state* s, int face, int ax, int64_t c, int i,
                               double fstar, double rhop) {
    const orc_face* f = &s->p.face[face];
    const int64_t V = s->V;
    if (f->ubc == ORC_U_PERIODIC) return;
    if (f->ubc == ORC_U_SPECULAR) { s->f_new[SPEC[ax][i] * V + c] = fstar; return; }
    const double Uw0 = f->ubc == ORC_U_MOVING ? f->uw[0] : 0.0;
    const double Uw1 = f->ubc == ORC_U_MOVING ? f->uw[1] : 0.0;
    const double Uw2 = f->ubc == ORC_U_MOVING ? f->uw[2] : 0.0;
    const int m = OPP[i];
    const double edu = (double)EX[m] * Uw0 + (double)EY[m] * Uw1 + (double)EZ[m] * Uw2;
    s->f_new[m * V + c] = fstar + 6.0 * rhop * W[m] * edu;
}

static void lbm_step(orc_state* s) {
    const orc_params* p = &s->p;
    const int64_t V = s->V;
    const double DT = p->DT, om = s->omega, omp = s->omega_prime, omf = s->omega_forcing;
    const int xlp = uper(p, 0), xhp = uper(p, 1), ylp = uper(p, 2), yhp = uper(p, 3);
    const int zlp = uper(p, 4), zhp = uper(p, 5);
#pragma omp parallel for schedule(static)
    for (int z = 0; z < p->nz; ++z)
        for (int y = 0; y < p->ny; ++y)
            for (int x = 0; x < p->nx; ++x) {
                const int64_t c = cidx(p, x, y, z);
                const double Fx = s->F[0][c], Fy = s->F[1][c], Fz = s->F[2][c];
                /* ComputeMoments (src/physics_helpers.h:92-121) */
                double rhop = 0.0, uxp = 0.0, uyp = 0.0, uzp = 0.0;
                for (int i = 0; i < 15; ++i) {
                    const double fi = s->f[i * V + c];
                    rhop += fi;
                    uxp += EX[i] * fi;
                    uyp += EY[i] * fi;
                    uzp += EZ[i] * fi;
                }
                uxp += 0.5 * Fx * DT;
                uyp += 0.5 * Fy * DT;
                uzp += 0.5 * Fz * DT;
                uxp /= rhop;
                uyp /= rhop;
                uzp /= rhop;
                s->rho[c] = rhop;
                s->u[0][c] = uxp;
                s->u[1][c] = uyp;
                s->u[2][c] = uzp;
                const double uF = uxp * Fx + uyp * Fy + uzp * Fz;
                const double u2 = uxp * uxp + uyp * uyp + uzp * uzp;
                for (int i = 0; i < 15; ++i) {
                    const double ex = (double)EX[i], ey = (double)EY[i], ez = (double)EZ[i];
                    /* ComputeFeqAndForcing (src/physics_helpers.h:73-90) */
                    const double ue = uxp * ex + uyp * ey + uzp * ez;
                    const double eF = ex * Fx + ey * Fy + ez * Fz;
                    const double feq = (W[i] * rhop * (1.0 + 3.0 * ue + 4.5 * ue * ue - 1.5 * u2));
                    const double forcing = omf * W[i] * (3.0 * eF - 3.0 * uF + 9.0 * ue * eF);
                    /* PointwiseBGKCollide (src/physics_helpers.h:123-129) */
                    const double fstar = om * s->f[i * V + c] + omp * feq + DT * forcing;
                    const int dx = stream_off(xlp, xhp, x, EX[i], p->nx);
                    const int dy = stream_off(ylp, yhp, y, EY[i], p->ny);
                    const int dz = stream_off(zlp, zhp, z, EZ[i], p->nz);
                    const int xc = dx < 0 || dx >= p->nx;
                    const int yc = dy < 0 || dy >= p->ny;
                    const int zc = dz < 0 || dz >= p->nz;
                    if (!xc && !yc && !zc) {
                        s->f_new[i * V + cidx(p, dx, dy, dz)] = fstar;
                    } else {
                        if (dx < 0) handle_wall(s, 0, 0, c, i, fstar, rhop);
                        else if (dx >= p->nx) handle_wall(s, 1, 0, c, i, fstar, rhop);
                        if (dy < 0) handle_wall(s, 2, 1, c, i, fstar, rhop);
                        else if (dy >= p->ny) handle_wall(s, 3, 1, c, i, fstar, rhop);
                        if (dz < 0) handle_wall(s, 4, 2, c, i, fstar, rhop);
                        else if (dz >= p->nz) handle_wall(s, 5, 2, c, i, fstar, rhop);
                    }
                }
            }
    double* t = s->f; s->f = s->f_new; s->f_new = t;
}

void orc_lbm_step(orc_state* s) { lbm_step(s); }

/* ActiveNematicSim::Step on the CPU build (src/active_nematic.h:84-108). */
void orc_step(orc_state* s, int nsteps) {
    for (int n = 0; n < nsteps; ++n) {
        q_step_setup(s);
        body_force(s);
        lbm_step(s);
    }
}

/* ---------------------------------------------------------------------- */
/* Diagnostics                                                             */

/* NematicFreeEnergyDensity (src/analysis_fields.cc:38-57) */
static double fe_density(const orc_params* p, double Qxx, double Qxy, double Qxz, double Qyy,
                         double Qyz, double lxx, double lxy, double lxz, double lyy, double lyz) {
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
    const double QlQ = 2.0 * Qxx * lxx + 2.0 * Qyy * lyy + Qxx * lyy + Qyy * lxx +
                       2.0 * (Qxy * lxy + Qxz * lxz + Qyz * lyz);
    return 0.5 * p->A * TrQ2 + (p->B / 3.0) * TrQ3 + 0.25 * p->C * TrQ2 * TrQ2 - 0.5 * p->L * QlQ;
}

double orc_free_energy(const orc_params* p, const double* q5) {
    const int64_t V = (int64_t)p->nx * p->ny * p->nz;
    double total = 0.0;
    for (int z = 0; z < p->nz; ++z)
        for (int y = 0; y < p->ny; ++y)
            for (int x = 0; x < p->nx; ++x) {
                const int64_t c = cidx(p, x, y, z);
                const int xm = fetch_off(qper(p, 0), qper(p, 1), x, -1, p->nx);
                const int xp = fetch_off(qper(p, 0), qper(p, 1), x, +1, p->nx);
                const int ym = fetch_off(qper(p, 2), qper(p, 3), y, -1, p->ny);
                const int yp = fetch_off(qper(p, 2), qper(p, 3), y, +1, p->ny);
                const int zm = fetch_off(qper(p, 4), qper(p, 5), z, -1, p->nz);
                const int zp = fetch_off(qper(p, 4), qper(p, 5), z, +1, p->nz);
                double l[5], Q[5];
                for (int k = 0; k < 5; ++k) {
                    const double* q = q5 + k * V;
                    Q[k] = q[c];
                    l[k] = q[cidx(p, xp, y, z)] + q[cidx(p, xm, y, z)] + q[cidx(p, x, yp, z)] +
                           q[cidx(p, x, ym, z)] + q[cidx(p, x, y, zp)] + q[cidx(p, x, y, zm)] - 6.0 * Q[k];
                }
                total += fe_density(p, Q[0], Q[1], Q[2], Q[3], Q[4], l[0], l[1], l[2], l[3], l[4]);
            }
    return total;
}

void orc_log_reduce(const orc_params* p, const double* rho, const double* u3, double* upast3,
                    double out[8]) {
    const int64_t V = (int64_t)p->nx * p->ny * p->nz;
    const double *ux = u3, *uy = u3 + V, *uz = u3 + 2 * V;
    double *px_ = upast3, *py_ = upast3 + V, *pz_ = upast3 + 2 * V;
    double mass = 0.0, px = 0.0, py = 0.0, pz = 0.0, ke = 0.0, e1 = 0.0, e2 = 0.0, umax2 = 0.0;
    for (int64_t c = 0; c < V; ++c) {
        mass += rho[c];
        px += rho[c] * ux[c];
        py += rho[c] * uy[c];
        pz += rho[c] * uz[c];
        const double u2 = ux[c] * ux[c] + uy[c] * uy[c] + uz[c] * uz[c];
        ke += 0.5 * rho[c] * u2;
        if (u2 > umax2) umax2 = u2;
        e1 += (ux[c] - px_[c]) * (ux[c] - px_[c]) + (uy[c] - py_[c]) * (uy[c] - py_[c]) +
              (uz[c] - pz_[c]) * (uz[c] - pz_[c]);
        e2 += u2;
        px_[c] = ux[c]; py_[c] = uy[c]; pz_[c] = uz[c];
    }
    out[0] = mass; out[1] = px; out[2] = py; out[3] = pz;
    out[4] = ke; out[5] = e1; out[6] = e2; out[7] = umax2;
}

void orc_order_director(const orc_params* p, const double* q5, double* order, double* director) {
    const int64_t V = (int64_t)p->nx * p->ny * p->nz;
    for (int64_t c = 0; c < V; ++c) {
        const double Qxx = q5[c], Qxy = q5[V + c], Qxz = q5[2 * V + c], Qyy = q5[3 * V + c],
                     Qyz = q5[4 * V + c];
        /* HalfTrQ2 and DetQ (src/analysis_fields.cc:17-34) */
        const double pp = (Qxx * Qxx + Qxx * Qyy + Qyy * Qyy + Qxy * Qxy + Qxz * Qxz + Qyz * Qyz);
        const double qq = (-(Qxx + Qyy) * (Qxx * Qyy - Qxy * Qxy) - Qyy * Qxz * Qxz -
                           Qxx * Qyz * Qyz + 2 * Qxy * Qxz * Qyz);
        const double r = 2.0 * sqrt(pp / 3.0);
        double arg = 4 * qq / (r * r * r);
        arg = arg < -1.0 ? -1.0 : (1.0 < arg ? 1.0 : arg);
        const double S = r * cos(1.0 / 3.0 * acos(arg));
        double nx_ = Qxz * (Qyy - S) - Qxy * Qyz;
        double ny_ = Qyz * (Qxx - S) - Qxy * Qxz;
        double nz_ = Qxy * Qxy - (Qxx - S) * (Qyy - S);
        const double ninv = 1.0 / sqrt(nx_ * nx_ + ny_ * ny_ + nz_ * nz_);
        nx_ *= ninv; ny_ *= ninv; nz_ *= ninv;
        director[3 * c + 0] = nx_;
        director[3 * c + 1] = ny_;
        director[3 * c + 2] = nz_;
        order[c] = S;
    }
}

/* FlipN (src/analysis/defect_fields.cc:17-24) */
static inline int flipn(const double* a, const double* b) {
    return (a[0] * b[0] + a[1] * b[1] + a[2] * b[2]) <= 0.0;
}

/* One plaquette loop n1 -> n2 -> n3 -> n4 -> n1 with sign alignment. */
static int plaquette(const double* d1, const double* d2, const double* d3, const double* d4) {
    double n2[3] = {d2[0], d2[1], d2[2]}, n3[3] = {d3[0], d3[1], d3[2]}, n4[3] = {d4[0], d4[1], d4[2]};
    if (flipn(d1, n2)) { n2[0] = -n2[0]; n2[1] = -n2[1]; n2[2] = -n2[2]; }
    if (flipn(n2, n3)) { n3[0] = -n3[0]; n3[1] = -n3[1]; n3[2] = -n3[2]; }
    if (flipn(n3, n4)) { n4[0] = -n4[0]; n4[1] = -n4[1]; n4[2] = -n4[2]; }
    return flipn(n4, d1);
}

int64_t orc_winding(const orc_params* p, const double* dir, uint8_t* def_x, uint8_t* def_y,
                    uint8_t* def_z) {
    const int nx = p->nx, ny = p->ny, nz = p->nz;
    int64_t count = 0;
#define D(x, y, z) (dir + 3 * cidx(p, (x), (y), (z)))
    for (int z = 0; z < nz - 1; ++z)
        for (int y = 0; y < ny - 1; ++y)
            for (int x = 0; x < nx; ++x) {
                const int fl = plaquette(D(x, y, z), D(x, y + 1, z), D(x, y + 1, z + 1), D(x, y, z + 1));
                def_x[((int64_t)z * (ny - 1) + y) * nx + x] = (uint8_t)fl;
                count += fl;
            }
    for (int z = 0; z < nz - 1; ++z)
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx - 1; ++x) {
                const int fl = plaquette(D(x, y, z), D(x + 1, y, z), D(x + 1, y, z + 1), D(x, y, z + 1));
                def_y[((int64_t)z * ny + y) * (nx - 1) + x] = (uint8_t)fl;
                count += fl;
            }
    for (int z = 0; z < nz; ++z)
        for (int y = 0; y < ny - 1; ++y)
            for (int x = 0; x < nx - 1; ++x) {
                const int fl = plaquette(D(x, y, z), D(x + 1, y, z), D(x + 1, y + 1, z), D(x, y + 1, z));
                def_z[((int64_t)z * (ny - 1) + y) * (nx - 1) + x] = (uint8_t)fl;
                count += fl;
            }
#undef D
    return count;
}

/* ---------------------------------------------------------------------- */
/* Seeded initial condition (this project's own generator)                 */

static inline uint64_t splitmix64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
/* Uniform in (0, 1) from counter (key, cell, k). */
static inline double uni(uint64_t key, uint64_t cell, uint64_t k) {
    const uint64_t h = splitmix64(key + cell * 16u + k);
    return ((double)(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}

void orc_seeded_q(const orc_params* p, uint64_t seed, double S0, double sigma, double* q5) {
    const int64_t V = (int64_t)p->nx * p->ny * p->nz;
    const uint64_t key = splitmix64(seed ^ 0x5851f42d4c957f2dULL);
    const double two_pi = 6.283185307179586476925286766559;
    /* Each cell depends on (seed, cell) only: any thread split gives the same field. */
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < V; ++c) {
        const double ct = 2.0 * uni(key, (uint64_t)c, 0) - 1.0;
        const double ph = two_pi * uni(key, (uint64_t)c, 1);
        const double st = sqrt(fmax(0.0, 1.0 - ct * ct));
        const double n0 = st * cos(ph), n1 = st * sin(ph), n2 = ct;
        double g[6];
        for (int k = 0; k < 3; ++k) {
            const double r = sqrt(-2.0 * log(uni(key, (uint64_t)c, 2 + 2 * k)));
            const double t = two_pi * uni(key, (uint64_t)c, 3 + 2 * k);
            g[2 * k] = r * cos(t);
            g[2 * k + 1] = r * sin(t);
        }
        q5[c] = S0 * (n0 * n0 - 1.0 / 3.0) + sigma * g[0];
        q5[V + c] = S0 * (n0 * n1) + sigma * g[1];
        q5[2 * V + c] = S0 * (n0 * n2) + sigma * g[2];
        q5[3 * V + c] = S0 * (n1 * n1 - 1.0 / 3.0) + sigma * g[3];
        q5[4 * V + c] = S0 * (n1 * n2) + sigma * g[4];
    }
}
