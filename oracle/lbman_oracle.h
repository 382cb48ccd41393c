/*
 * lbman_oracle.h -- CPU restatement of lbman3d's per-timestep hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * implementation in lbman3d_b200/: only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg may load it.  No product code path calls it.
 *
 * It restates, in plain C with runtime parameters, the FP64 algorithm of the
 * reference CPU solver (src/lbm_solver.tpp, src/qtensor_solver.tpp,
 * src/model.h, src/physics_helpers.h, src/boundary_handler.h, src/offsets.h,
 * src/analysis_fields.{h,cc}, src/analysis/defect_finder.tpp, src/sim_io.cc).
 * Every arithmetic expression keeps the reference's association order, and
 * the library is compiled with -ffp-contract=off, so results are bitwise
 * equal to the reference compiled with g++ -O3 on x86-64.  The pin against
 * the reference itself is tests/golden/ (fixtures written by
 * oracle/ref_driver.cc built from the reference sources).
 *
 * Layout: structure of arrays, x fastest, cell = (z*ny + y)*nx + x, and
 * populations direction-major f[i*V + cell] (the reference's device layout,
 * src/local_grid.h:64).  Vectors (u, force) are passed as 3 consecutive
 * blocks of V values; Q as 5 blocks (xx, xy, xz, yy, yz).
 */
#ifndef LBMAN_ORACLE_H_
#define LBMAN_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_Q_PERIODIC = 0, ORC_Q_NEUMANN = 1, ORC_Q_ANCHORING = 2 };
enum { ORC_U_PERIODIC = 0, ORC_U_NOSLIP = 1, ORC_U_MOVING = 2, ORC_U_SPECULAR = 3 };
enum { ORC_CENTRED = 0, ORC_UPWIND = 1 };

typedef struct {
    int qbc;                 /* ORC_Q_*                                      */
    double s, theta, phi;    /* Anchoring<S, theta, phi>                     */
    int ubc;                 /* ORC_U_*                                      */
    double uw[3];            /* MovingWall<Ux, Uy, Uz>                       */
} orc_face;

typedef struct {
    int nx, ny, nz;
    double DT, kDensity, TAUF, L, A, B, C, LAMBDA, GAMMA, ALPHA, MU;
    int advection;           /* ORC_CENTRED / ORC_UPWIND                     */
    orc_face face[6];        /* XLo, XHi, YLo, YHi, ZLo, ZHi                 */
} orc_params;

typedef struct orc_state orc_state;

void orc_params_default(orc_params* p);
/* AnchoredQ<Anchoring<S,theta,phi>> (src/boundary_handler.h:232-251).      */
void orc_anchored_q(const orc_face* f, double out[5]);
double orc_equilibrium_order(const orc_params* p);

orc_state* orc_new(const orc_params* p);
void orc_free(orc_state* s);
/* Load fields.  f == NULL: f = f_eq(rho, u) (LbmSolver::Initialize).
 * force == NULL: zero body force.                                          */
void orc_set(orc_state* s, const double* rho, const double* u3, const double* q5,
             const double* f15, const double* force3);
/* Read fields back; any pointer may be NULL.                               */
void orc_get(const orc_state* s, double* rho, double* u3, double* q5, double* f15,
             double* force3, double* sigma5, double* tau3);
/* QTensorSolver::Step then LbmSolver::LatticeBoltzmannStep, n times.       */
void orc_step(orc_state* s, int nsteps);
/* QTensorSolver::Step (StepAndSetupBodyForce + SetActiveStressAndCompute-
 * BodyForce).  with_active == 0 mimics a subclass whose
 * SetActiveStressAndComputeBodyForce is empty (the reference tests'
 * ZeroActivitySolver).                                                    */
void orc_q_step(orc_state* s, int with_active);
/* LbmSolver::LatticeBoltzmannStep with the current body force.            */
void orc_lbm_step(orc_state* s);

/* Diagnostics ------------------------------------------------------------ */
/* TotalNematicFreeEnergy<BC> (src/analysis_fields.h:39-72), sequential sum. */
double orc_free_energy(const orc_params* p, const double* q5);
/* SimIO::Log sums (src/sim_io.cc:83-108): out = {mass, px, py, pz, ke, e1,
 * e2, umax2}.  upast3 is updated in place like AnalysisFields::u*_past_.   */
void orc_log_reduce(const orc_params* p, const double* rho, const double* u3,
                    double* upast3, double out[8]);
/* QtensorToOrderDirector (src/analysis_fields.cc:59-93): order[V],
 * director[3V] AoS (cell*3 + c).                                          */
void orc_order_director(const orc_params* p, const double* q5, double* order,
                        double* director);
/* DefectFinder::ComputeWindingNumbers (src/analysis/defect_finder.tpp:13-165):
 * def_x[nx*(ny-1)*(nz-1)], def_y[(nx-1)*ny*(nz-1)], def_z[(nx-1)*(ny-1)*nz].
 * Returns the number of flagged faces.                                    */
int64_t orc_winding(const orc_params* p, const double* director, uint8_t* def_x,
                    uint8_t* def_y, uint8_t* def_z);

/* Seeded initial condition used by every workload of this project:
 * Q = S0 (n n^T - I/3) with n uniform on the sphere per cell, plus
 * N(0, sigma^2) on each of the 5 stored components.  Counter based
 * (splitmix64 of seed and cell index), so any sub-box can be regenerated. */
void orc_seeded_q(const orc_params* p, uint64_t seed, double S0, double sigma,
                  double* q5);

#ifdef __cplusplus
}
#endif
#endif
