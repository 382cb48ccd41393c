/*
 * lbman3d.h -- C ABI of the B200 (sm_100a) implementation of lbman3d's
 * per-timestep hot path: the D3Q15 lattice-Boltzmann collide/stream, the
 * Beris-Edwards Q-tensor step with the active/passive body force, every wall
 * rule of the reference, and the diagnostic reductions.
 *
 * Plain C: pointers, sizes and int status codes, no C++ or torch types.
 * Host buffers are always float64 in the reference's host layout
 * (x fastest, cell = (z*ny + y)*nx + x); vector fields are 3 consecutive
 * blocks of V = nx*ny*nz values, Q is 5 blocks (xx, xy, xz, yy, yz) and
 * populations are 15 blocks, direction-major (f[i*V + cell], the
 * reference's device layout, src/local_grid.h:64).  Device memory is owned by
 * the library; host memory by the caller.
 *
 * Every entry point returns LBMAN_OK (0) or an error code; lbman_last_error()
 * gives a message for the calling thread.  A thin C++ layer
 * (include/lbman3d_dropin.hpp) maps the reference's DeviceFields /
 * DeviceSolver<BC> / LbmSolver<BC> / QTensorSolver<BC> onto these calls and
 * throws std::runtime_error on a non-zero status, the reference's error
 * convention (src/cuda/cuda_utils.h:5-10).
 */
#ifndef LBMAN3D_H_
#define LBMAN3D_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBMAN_ABI_VERSION 1

/* Status codes. */
#define LBMAN_OK 0
#define LBMAN_ERR_ARG 1         /* invalid argument or configuration            */
#define LBMAN_ERR_CUDA 2        /* a CUDA call failed                            */
#define LBMAN_ERR_DIVERGED 3    /* NaN in the global mass or momentum            */
#define LBMAN_ERR_TIMEOUT 4     /* a bounded device wait gave up                 */
#define LBMAN_ERR_STATE 5       /* call out of order (e.g. step before upload)   */
#define LBMAN_ERR_UNSUPPORTED 6 /* configuration this library does not implement */
#define LBMAN_ERR_NOMEM 7       /* device allocation failed                      */

/* Q-tensor wall tags (src/boundary.h:31-42). */
#define LBMAN_Q_PERIODIC 0
#define LBMAN_Q_NEUMANN 1
#define LBMAN_Q_ANCHORING 2
/* Velocity wall tags (src/boundary.h:31-50). */
#define LBMAN_U_PERIODIC 0
#define LBMAN_U_NOSLIP 1
#define LBMAN_U_MOVING 2
#define LBMAN_U_SPECULAR 3
/* Advection scheme (src/qtensor_types.h:19, kQAdvection). */
#define LBMAN_CENTRED 0
#define LBMAN_UPWIND 1
/* Storage / compute precision. */
#define LBMAN_FP64 0 /* FP64 compute and storage, the reference's arithmetic   */
#define LBMAN_FP32 1 /* FP32 compute, populations stored as f_i - w_i*rho0    */
#define LBMAN_FP16 2 /* FP32 compute, populations stored as FP16 deviations   */
/* Kernel organisation. */
#define LBMAN_KERNELS_AUTO 0
#define LBMAN_KERNELS_SPLIT 1 /* Q+force kernel, then LBM kernel               */
#define LBMAN_KERNELS_FUSED 2 /* one kernel per time step                      */
#define LBMAN_KERNELS_SPLIT_PAIR 3 /* split, the Q+force kernel updating two
                                 points per thread with packed FP32 pairs
                                 (FP32/FP16 precision; tiles 30x6, 30x10,
                                 30x14; nx a multiple of 4)                  */

/* One face of the box: WallSpec<QBC, UBC> (src/boundary.h:72-76). */
typedef struct lbman_face {
    int qbc;                  /* LBMAN_Q_*                                  */
    double s, theta, phi;     /* Anchoring<S, theta, phi> (radians)          */
    int ubc;                  /* LBMAN_U_*                                  */
    double uw[3];             /* MovingWall<Ux, Uy, Uz>                      */
} lbman_face;

/* Runtime form of params.h + sim_config.h + the BC type (SimBC). */
typedef struct lbman_config {
    int nx, ny, nz;
    double DT, kDensity, TAUF, L, A, B, C, LAMBDA, GAMMA, ALPHA, MU;
    int advection;            /* LBMAN_CENTRED / LBMAN_UPWIND                */
    lbman_face face[6];       /* XLo, XHi, YLo, YHi, ZLo, ZHi                */
    int precision;            /* LBMAN_FP64 / LBMAN_FP32 / LBMAN_FP16        */
    int kernels;              /* LBMAN_KERNELS_*                             */
    int device;               /* CUDA device ordinal                         */
    int tile_x, tile_y, zchunk, threads; /* 0 = library default           */
} lbman_config;

/* Global diagnostics (src/sim_io.cc:78-166, src/analysis_fields.h:39-72). */
typedef struct lbman_diag {
    double mass, px, py, pz;  /* sum rho, sum rho*u                          */
    double kinetic_energy;    /* sum rho*|u|^2/2                             */
    double rel_change_num;    /* sum |u - u_prev|^2 since the previous call  */
    double rel_change_den;    /* sum |u|^2                                   */
    double umax2;             /* max |u|^2                                   */
    double free_energy;       /* TotalNematicFreeEnergy (LBMAN_DIAG_ENERGY)  */
    int64_t defect_faces;     /* plaquettes with a director sign flip
                                 (LBMAN_DIAG_DEFECTS), -1 if not computed    */
    int nan_detected;         /* NaN in mass or momentum                     */
} lbman_diag;

#define LBMAN_DIAG_FLOW 1     /* mass, momentum, kinetic energy, max |u|       */
#define LBMAN_DIAG_ENERGY 2   /* nematic free energy                          */
#define LBMAN_DIAG_DEFECTS 4  /* director sign-flip plaquette count           */
#define LBMAN_DIAG_ALL 7

typedef struct lbman_solver lbman_solver;

/* params.h defaults (src/params.h:14-112), SimBC = SlitNoSlipConfig, FP64. */
int lbman_config_init(lbman_config* cfg);
const char* lbman_status_string(int status);
const char* lbman_last_error(void);
int lbman_abi_version(void);

/* Device description, InitializeComputeBackend (src/device_fields.h:21). */
int lbman_device_info(int device, char* buf, size_t len);

/* DeviceFields(LocalGrid) + DeviceSolver<BC>::Initialize
 * (src/device_fields.h:174, src/device_solver.h:15).  Rejects an axis whose
 * velocity tag is periodic on one face only.                                */
int lbman_create(const lbman_config* cfg, lbman_solver** out);
int lbman_destroy(lbman_solver* s);
/* Issue all work on this cudaStream_t (default: a stream owned by s).        */
int lbman_set_stream(lbman_solver* s, void* cuda_stream);
int lbman_synchronize(lbman_solver* s);

/* DeviceFields::Initialize(FluidFields&, const QTensorFields&)
 * (src/device_fields.h:179).  rho[V], u3[3V], q5[5V] required; f15 (15V,
 * direction-major) NULL means f = f_eq(rho, u) as LbmSolver::Initialize
 * (src/lbm_solver.tpp:35-62); force3 NULL means zero body force.            */
int lbman_upload(lbman_solver* s, const double* rho, const double* u3, const double* q5,
                 const double* f15, const double* force3);
/* Seeded initial state generated on the device (no host transfer): rho =
 * kDensity, u = 0, zero body force, Q = S0 (n n^T - I/3) with n uniform on
 * the sphere per cell plus N(0, sigma^2) on each stored Q component
 * (counter-based splitmix64 of seed and cell index), f = f_eq.  This is the
 * initial condition of every benchmark workload; it replaces the
 * reference's unseeded QTensorSolver::Initialize
 * (src/qtensor_solver.tpp:14-48) the way its tests override Initialize.    */
int lbman_init_seeded(lbman_solver* s, uint64_t seed, double S0, double sigma);

/* DeviceFields::CopyToHost (src/device_fields.h:181); any pointer may be NULL.
 * f15 receives the pre-collision populations, as the reference stores them. */
int lbman_download(lbman_solver* s, double* rho, double* u3, double* q5, double* f15,
                   double* force3);

/* ActiveNematicSim::Step (src/active_nematic.h:104-108), n times.            */
int lbman_step(lbman_solver* s, int nsteps);
/* DeviceSolver<BC>::QTensorStep: Q update + full body force
 * (src/cuda/device_solver.cu:35-98).                                         */
int lbman_qtensor_step(lbman_solver* s);
/* DeviceSolver<BC>::LBMStep: collide + stream + walls with the current body
 * force (src/cuda/device_solver.cu:101-121).                                 */
int lbman_lbm_step(lbman_solver* s);

/* The Q stage as the reference's two phases, for callers that replace the
 * activity model between them (a subclass overriding the virtual
 * QTensorSolver::SetActiveStressAndComputeBodyForce, src/qtensor_solver.h:
 * 11-21, 48).  lbman_qtensor_step does both in one pass.
 *   lbman_qtensor_setup  <- QTensorSolver::StepAndSetupBodyForce
 *                           (src/qtensor_solver.tpp:51-147): Q := Q_new, the
 *                           stresses Sigma (5) and tau (3) kept on the device,
 *                           body force := the Ericksen seed.
 *   lbman_active_force   <- the base SetActiveStressAndComputeBodyForce
 *                           (src/qtensor_solver.tpp:155-217): body force +=
 *                           -ALPHA div Q + div(Sigma + tau) - MU u.
 *   lbman_download_stress / lbman_upload_stress: Sigma [5V] (xx xy xz yy yz)
 *                           and tau [3V] (xy xz yz), FP64 host arrays
 *                           (QTensorFields::Sigma_* / Tau_*).               */
int lbman_qtensor_setup(lbman_solver* s);
int lbman_active_force(lbman_solver* s);
int lbman_download_stress(lbman_solver* s, double* sigma5, double* tau3);
int lbman_upload_stress(lbman_solver* s, const double* sigma5, const double* tau3);

/* SimIO::Log reductions + TotalNematicFreeEnergy + defect plaquettes, FP64
 * accumulation on the device.  Returns LBMAN_ERR_DIVERGED (after filling out)
 * when the mass or momentum is NaN, as SimIO::Log returns false.            */
int lbman_reduce(lbman_solver* s, int flags, lbman_diag* out);

/* Flow diagnostics without any device allocation.  No counterpart in the
 * reference: it is an addition for callers that cannot call cudaMalloc --
 * a host framework whose allocator already holds (nearly) all device memory,
 * or a stepping loop that must not allocate or free because cudaFree
 * synchronises the whole device.
 *
 * Computes what lbman_reduce(LBMAN_DIAG_FLOW) computes (mass, momentum,
 * kinetic energy, relative change against upast3, max |u|^2, NaN check) over
 * caller-owned device fields: rho[ncells] and u3[3*ncells] (double when
 * precision is LBMAN_FP64, float when LBMAN_FP32), upast3[3*ncells] of the same
 * type, read and then overwritten with u3.  Work is issued on cuda_stream
 * (NULL: the legacy default stream) on the current device, and the call
 * returns after the result is copied into *out.
 *
 * Scratch comes from a fixed array inside the library (partial sums of at
 * most LBMAN_NOALLOC_MAX_BLOCKS blocks, about 76 KB per device, held by every
 * GPU that loads the library until the process exits).  Each call looks up
 * that array's device address in the current device's context.  The call
 * copies its result to the host and synchronises cuda_stream, so it cannot be
 * issued while that stream is being captured.  All calls share the array:
 * calls whose GPU work overlaps (other streams or threads, same device) race
 * and corrupt each other's results; serialise them.  A CUDA error already
 * pending on the calling thread is reported (LBMAN_ERR_CUDA) and left
 * pending.  ncells above LBMAN_NOALLOC_MAX_CELLS is rejected with
 * LBMAN_ERR_ARG.  Allocates nothing: no cudaMalloc, no cudaFree, no
 * allocating library call.                                                  */
#define LBMAN_NOALLOC_MAX_BLOCKS 1184
#define LBMAN_NOALLOC_MAX_CELLS 2147483647LL
int lbman_flow_reduce_noalloc(int64_t ncells, int precision, const void* rho, const void* u3,
                              void* upast3, void* cuda_stream, lbman_diag* out);

/* Launch shape of the time step: kernel organisation and z-marching tile.   */
typedef struct lbman_shape {
    int kernels;              /* LBMAN_KERNELS_SPLIT / _FUSED / _SPLIT_PAIR   */
    int tile_x, tile_y;       /* cells per x-y plane of one block             */
    int zchunk;               /* > 0: z planes marched by one block;
                                 <= 0: balanced schedule, max(1, -zchunk)
                                 waves of resident blocks, each taking an
                                 equal share of the column planes            */
    int threads;              /* threads per block (set by the tile)          */
    double ms_per_step;       /* measured by lbman_autotune, else 0           */
    int blocks;               /* blocks of the Q+force (or fused) launch of a
                                 solver; 0 from the ensemble calls           */
} lbman_shape;

int lbman_get_shape(lbman_solver* s, lbman_shape* out);
/* Select a shape (tile_x x tile_y must be one of the compiled tiles: 30x6,
 * 32x6, 14x14, 32x8, and for FP32/FP16 also 30x14, 62x6, 32x14, 64x6;
 * zchunk >= -8).                                                           */
int lbman_set_shape(lbman_solver* s, const lbman_shape* shape);
/* Autotuner (no counterpart in the reference): times steps_per_trial steps
 * of every kernel organisation x compiled tile x z-chunk candidate on the
 * current state with CUDA events, keeps the fastest and restores the state
 * it started from bit for bit (a temporary device copy of the fields is
 * taken for that).  ntrials (may be NULL) receives the number of candidates
 * timed.                                                                    */
int lbman_autotune(lbman_solver* s, int steps_per_trial, lbman_shape* best, int* ntrials);

/* z-slab decomposition of one box across GPUs (or across handles on one GPU).
 * Replaces the reference's MPI domain decomposition (src/mpi/mpi_context.h,
 * src/mpi/halo_exchange_qtensor.h:131-209, src/mpi/halo_exchange_lbm.h:
 * 304-386) for the single split axis z.
 *
 * lbman_create_slab makes a handle that owns planes [z_offset, z_offset +
 * cfg->nz) of a box of nz_global planes (cfg->nz >= 2).  The box's z faces
 * must be periodic (every reference preset: FullyPeriodic, Channel, Slit,
 * SlitNoSlip); x and y keep any wall.  The handle allocates two ghost planes
 * on each side and steps with the in-place organisations (LBMAN_KERNELS_SPLIT
 * or _SPLIT_PAIR; AUTO means SPLIT).  upload / download / init_seeded take
 * the owned planes (V = nx*ny*cfg->nz); init_seeded gives the owned planes
 * of the whole box's seeded field.  Slabs i-1 and i+1 (mod the slab count)
 * are the neighbours across the low and high z face.
 *
 * A step is three exchanges around the two kernel calls:
 *   exchange LBMAN_HALO_QU; lbman_qtensor_step;
 *   exchange LBMAN_HALO_F_IN; lbman_lbm_step; exchange LBMAN_HALO_F_OUT.
 * The Q+force kernel computes the passive stresses of the ghost planes
 * itself from the 2-deep Q/u halo, so no stress halo is exchanged.  The
 * population exchanges move the 5 crossing directions of one plane and only
 * around odd in-place steps (even steps are local); lbman_halo_spans returns
 * n = 0 when the phase has nothing to move.  F_OUT lands in a staging area
 * and lbman_halo_done merges it, keeping the slots that this slab's own
 * x / y wall rule wrote (the reference's unpack skip rule).  Calls out of
 * this order return LBMAN_ERR_STATE; lbman_step and the two-phase Q stage
 * are not available on slabs; lbman_reduce on a slab sums its owned planes
 * (LBMAN_DIAG_ENERGY needs a fresh QU halo; defects are not counted).      */
#define LBMAN_HALO_QU 0    /* Q (5), u (3): 2 owned planes -> neighbour ghosts  */
#define LBMAN_HALO_F_IN 1  /* 5 populations: owned plane -> neighbour ghost     */
#define LBMAN_HALO_F_OUT 2 /* 5 populations: ghost plane -> neighbour's owned   */
#define LBMAN_HALO_MAX_SPANS 8

#define LBMAN_FIELD_Q 0      /* component 0-4 of the current Q              */
#define LBMAN_FIELD_U 1      /* component 0-2 of the current velocity       */
#define LBMAN_FIELD_F 2      /* population slot 0-14 (stored form)          */
#define LBMAN_FIELD_FSTAGE 3 /* F_OUT staging: slot 0-4 of face `plane`     */

/* One contiguous span of an exchange: `planes` planes of one component,
 * starting at `plane` in owned coordinates (owned 0 .. nz_local-1, ghosts
 * -2, -1 and nz_local, nz_local+1).                                        */
typedef struct {
    int field;
    int comp;
    int plane;
    int planes;
} lbman_halo_span;

int lbman_create_slab(const lbman_config* cfg, int nz_global, int z_offset, lbman_solver** out);
/* The spans of an exchange phase for a slab of nz_local planes (host only).
 * send[f][k] goes to the neighbour across face f (0 = low z, 1 = high z),
 * which receives it into its recv[1-f][k]; n spans per face (8 for QU, 5 for
 * the population phases).                                                   */
int lbman_halo_plan(int nz_local, int phase, lbman_halo_span send[2][LBMAN_HALO_MAX_SPANS],
                    lbman_halo_span recv[2][LBMAN_HALO_MAX_SPANS], int* n);
/* The plan's spans as device addresses of this slab's current buffers, all
 * span_bytes long; n = 0 when the phase moves nothing now.  A transport
 * (NCCL send/recv, peer copies) delivers them, then calls lbman_halo_done. */
int lbman_halo_spans(lbman_solver* s, int phase, void* send[2][LBMAN_HALO_MAX_SPANS],
                     void* recv[2][LBMAN_HALO_MAX_SPANS], size_t* span_bytes, int* n);
int lbman_halo_done(lbman_solver* s, int phase);
/* In-process transport: slabs[0..n-1] in z order (same or different
 * devices), each slab's spans copied into its neighbours' with
 * cudaMemcpyAsync on the receivers' streams, ordered by events (no host
 * synchronisation), then lbman_halo_done on every slab.                    */
int lbman_slab_exchange(lbman_solver* const* slabs, int nslabs, int phase);
/* nz_global, z_offset, nz_local of a slab (0, 0, nz for a whole box).       */
int lbman_slab_info(lbman_solver* s, int* nz_global, int* z_offset, int* nz_local);

/* Ensemble runner (no counterpart in the reference, whose solver advances one
 * box per process).  Many independent boxes -- each with its own lbman_config
 * (size, boundary faces, physical parameters) -- advance together: every time
 * step is one launch per kernel covering all boxes (a persistent grid walking
 * a box/tile work list), and lbman_ensemble_step replays steps from a CUDA
 * graph.  All boxes share precision, advection scheme and device; the launch
 * shape comes from boxes[0] (kernels, tile_x/y, zchunk) or from
 * lbman_ensemble_autotune.  Each box's results are bitwise identical to
 * running it alone through lbman_step with the same precision.              */
typedef struct lbman_ensemble lbman_ensemble;
int lbman_ensemble_create(const lbman_config* boxes, int nboxes, lbman_ensemble** out);
int lbman_ensemble_destroy(lbman_ensemble* e);
int lbman_ensemble_set_stream(lbman_ensemble* e, void* cuda_stream);
/* Box b gets lbman_init_seeded's state with seed + b and S0 = its own
 * equilibrium order (src/model.h:39-41).                                    */
int lbman_ensemble_init_seeded(lbman_ensemble* e, uint64_t seed, double sigma);
/* The same with one seed per box (box b's field is a single box's
 * lbman_init_seeded(seeds[b]) field): a rank holding a share of a larger
 * ensemble seeds its boxes by their index in the whole ensemble.           */
int lbman_ensemble_init_seeded_each(lbman_ensemble* e, const uint64_t* seeds, double sigma);
/* Before the first step only: rho, u, Q of one box; f = f_eq, F = 0.       */
int lbman_ensemble_upload(lbman_ensemble* e, int box, const double* rho, const double* u3, const double* q5);
int lbman_ensemble_download(lbman_ensemble* e, int box, double* rho, double* u3, double* q5, double* f15);
int lbman_ensemble_step(lbman_ensemble* e, int nsteps);
int lbman_ensemble_synchronize(lbman_ensemble* e);
int lbman_ensemble_set_shape(lbman_ensemble* e, int kernels, int tile_x, int tile_y, int zchunk);
int lbman_ensemble_get_shape(lbman_ensemble* e, lbman_shape* out);
/* Times every kernel organisation x tile x z-chunk candidate over the whole
 * ensemble, keeps the fastest, restores every box's state bit for bit.     */
int lbman_ensemble_autotune(lbman_ensemble* e, int steps_per_trial, lbman_shape* best, int* ntrials);
int lbman_ensemble_info(lbman_ensemble* e, int64_t* cells, int64_t* steps, int64_t* launches);

/* Statistics of the current state (no counterpart in the reference, whose
 * analysis stops at the defect finder).  The first call allocates cuFFT
 * plans and scratch (about 5 x 8 x V bytes in FP64, half that otherwise),
 * kept until lbman_destroy.  Every axis is transformed as periodic.  Shell
 * sums are accumulated in FP64; 1 <= nbins <= 8192; shells beyond nbins are
 * dropped.                                                                  */
#define LBMAN_STATS_MAX_BINS 8192

/* Shell-averaged kinetic-energy spectrum: E[b] = (1 / 2V^2) sum of |u_hat(k)|^2
 * over the wavevectors of shell b = round(n_max |(m_x/nx, m_y/ny, m_z/nz)|),
 * m the integer wavenumbers (|m_a| <= n_a/2), n_max = max(nx, ny, nz);
 * sum_b E[b] = <|u|^2>/2 once nbins > n_max*sqrt(3)/2.  counts (may be NULL)
 * receives the number of wavevectors per shell.                            */
int lbman_velocity_spectrum(lbman_solver* s, int nbins, double* E, double* counts);

/* Radially averaged Q-tensor autocorrelation C[b] = <Q(x):Q(x+r)> / <Q:Q>
 * (full 3x3 contraction, qzz = -qxx - qyy), r binned by b = round(|r|) with
 * minimum-image separations; counts (may be NULL) receives the separations
 * per shell.  xi (may be NULL) receives the correlation length: the |r| at
 * which C first falls below 1/e, linearly interpolated between shells, or
 * -1 if it does not within nbins shells.                                    */
int lbman_q_correlation(lbman_solver* s, int nbins, double* C, double* counts, double* xi);

typedef struct lbman_stats {
    double mean_speed;        /* <|u|> over cells                              */
    double rms_speed;         /* sqrt(<|u|^2>)                                  */
    int64_t defect_faces;     /* as lbman_reduce(LBMAN_DIAG_DEFECTS), -1 if any
                                 side is below 2 cells                          */
    double defect_density;    /* defect_faces / V, -1 if not computed          */
} lbman_stats;
int lbman_statistics(lbman_solver* s, lbman_stats* out);

/* Learned closure (no counterpart in the reference).
 *
 * Tensor-core self-test: one 128x32x64 BF16 GEMM with FP32 accumulation
 * through tcgen05 for each of the four operand-major combinations (A, B each
 * K- or MN-major), compared with an FP64 host product of the same BF16
 * inputs.  max_rel_err[4] (may be NULL) receives max |D - D_ref| / sum |a b|
 * per combination (-1 if the device wait timed out).                       */
int lbman_closure_selftest(int device, double* max_rel_err);

/* The closure network: 4 periodic 3x3x3 convolutions, 9 -> 32 -> 32 -> 32 -> 8
 * channels, GELU after the first three; BF16 weights and activations, FP32
 * accumulation, forward and backward on tcgen05 tensor cores.  Inputs are
 * the coarse rho, u (3) and Q (5), normalised per channel by (x - shift) /
 * scale; outputs are corrections to Q (5) and u (3) in units of out_scale.
 * The handle owns the network for one coarse grid size, Adam state and a
 * device-resident training set of box-filtered fine snapshots.             */
typedef struct lbman_closure lbman_closure;
int lbman_closure_create(int device, int nx, int ny, int nz, uint64_t seed, lbman_closure** out);
int lbman_closure_destroy(lbman_closure* c);
/* Parameters as one FP32 vector: per layer W[27][cin][cout] (cin 16, 32,
 * 32, 32; cout 32, 32, 32, 16; tap = (dz+1)*9 + (dy+1)*3 + (dx+1)) then
 * b[cout]; padding entries (layer-0 inputs 9..15, layer-3 outputs 8..15)
 * are held at zero.                                                       */
int lbman_closure_param_count(void);
int lbman_closure_get_params(lbman_closure* c, float* params);
int lbman_closure_set_params(lbman_closure* c, const float* params);
int lbman_closure_get_scales(lbman_closure* c, float* shift9, float* scale9, float* out_scale8);
int lbman_closure_set_scales(lbman_closure* c, const float* shift9, const float* scale9, const float* out_scale8);
/* Network on host fields feat9 [9][V] (rho, u, Q); out8 [8][V] receives the
 * normalised outputs.                                                       */
int lbman_closure_forward(lbman_closure* c, const float* feat9, float* out8);
/* Loss (1/8V) sum_c sum_j (out_j - target_j / out_scale_j)^2 for raw targets
 * target8 [8][V], and its gradient with respect to every parameter
 * (grad may be NULL), without updating anything.                          */
int lbman_closure_gradient(lbman_closure* c, const float* feat9, const float* target8, double* loss, float* grad);
/* Appends the box-filtered state of an FP32/FP16 fine solver whose grid is
 * f times the closure grid on every axis; new_trajectory starts a new
 * sequence (pairs never span two sequences).                              */
int lbman_closure_record(lbman_closure* c, lbman_solver* fine, int new_trajectory);
/* The same from box `box` of an ensemble (the training data of many fine
 * runs advanced together), as a snapshot of trajectory `trajectory` (>= 0,
 * the caller's id; one id per box).                                        */
int lbman_closure_record_box(lbman_closure* c, lbman_ensemble* e, int box, int trajectory);
int lbman_closure_dataset(lbman_closure* c, int* snapshots, int* pairs);
/* For each snapshot k and the next snapshot k' of its trajectory, the target
 * snapshot(k') - coarse_step(snapshot k), where coarse_step rebuilds the
 * populations as f_eq and takes one step of the coarse solver (FP32/FP16 on
 * the closure grid, with the coarse-grid parameters).  fit_scales sets the
 * input shift/scale to the per-channel mean/std of the snapshots and the
 * output scales to the rms target of Q and of u.                          */
int lbman_closure_build_targets(lbman_closure* c, lbman_solver* coarse, int fit_scales);
/* Rollout ("pushforward") pairs: from every stride-th snapshot k that has a
 * snapshot k'' m + 1 recordings later in its trajectory, m corrected coarse
 * steps with the current network give the state x the corrected run is in;
 * the pair is (x, snapshot(k'') - coarse_step(x)).  Training on them teaches
 * the network to correct its own accumulated error.  Appended to the pairs
 * of lbman_closure_build_targets (which clears both); *added receives the
 * count.                                                                   */
int lbman_closure_add_rollout_pairs(lbman_closure* c, lbman_solver* coarse, int m, int stride, int* added);
/* Adam (beta 0.9 / 0.999) on random training pairs; loss_first/last receive
 * the mean loss of the first and last tenth of the iterations.            */
int lbman_closure_train(lbman_closure* c, int iters, float lr, uint64_t seed, double* loss_first, double* loss_last);
/* train_noise: std of Gaussian noise added to the normalised network inputs
 * during lbman_closure_train (0 = none, the default); gain: multiplier of the
 * correction in lbman_closure_step (1 = default).                          */
int lbman_closure_set_options(lbman_closure* c, float train_noise, float gain);
/* Polls of each tensor-core completion wait of the closure's kernels before
 * the wait gives up (default LBMAN_CLOSURE_WAIT_DEFAULT).  A wait that gives
 * up makes the call return LBMAN_ERR_TIMEOUT; the kernel still lets every
 * MMA it issued finish (that drain keeps the default limit) before it frees
 * its tensor memory, so the next call runs normally.  0 makes the first
 * completion wait of every CTA give up: a way to exercise the timeout path.
 * No counterpart in the reference.                                          */
#define LBMAN_CLOSURE_WAIT_DEFAULT 67108864u
int lbman_closure_set_wait_limit(lbman_closure* c, uint32_t polls);
/* Coarse solver state := snapshot k.                                        */
int lbman_closure_load_snapshot(lbman_closure* c, int k, lbman_solver* coarse);
/* nsteps corrected coarse steps: network on the current state, populations
 * rebuilt as f_eq, one solver step, then Q and u corrected.               */
int lbman_closure_step(lbman_closure* c, lbman_solver* coarse, int nsteps);

/* Disclination lines (the reference's DefectFinder::FindDefects,
 * src/analysis/defect_finder.tpp): plaquette defect flags of the current Q on
 * the device, then on the host the face connectivity graph and its
 * decomposition into paths, as the reference builds them (same sweep order,
 * same unordered-map / ordered-set graph, same greedy walk), so the lines and
 * their count equal the reference's.  points (may be NULL) receives the face
 * centres of every path, xyz, while 3 * (points so far) <= points_cap;
 * line_offsets (may be NULL) receives the start of each path in points
 * (line_offsets[0] = 0, then one entry per path, while the index < cap).
 * Call once with NULL buffers to size them.  Every side needs >= 2 cells.  */
typedef struct lbman_defects {
    int64_t faces;            /* flagged plaquettes                           */
    int64_t edges;            /* graph edges                                  */
    int64_t lines;            /* paths (the reference's disclinations)        */
    int64_t points;           /* path vertices over all lines                 */
} lbman_defects;
int lbman_defect_lines(lbman_solver* s, lbman_defects* info, double* points, int64_t points_cap,
                       int64_t* line_offsets, int64_t offsets_cap);
/* The same graph and paths from host flag arrays (def_x nx*(ny-1)*(nz-1),
 * def_y (nx-1)*ny*(nz-1), def_z (nx-1)*(ny-1)*nz, x fastest, 1 = flagged);
 * qper6[f] != 0 when face f's Q tag is periodic (QXoff wraps there).  Host
 * only.                                                                     */
int lbman_defect_graph(int nx, int ny, int nz, const int* qper6, const uint8_t* def_x, const uint8_t* def_y,
                       const uint8_t* def_z, lbman_defects* info, double* points, int64_t points_cap,
                       int64_t* line_offsets, int64_t offsets_cap);

/* Steps completed since the last upload. */
int lbman_steps_done(lbman_solver* s, int64_t* steps);
/* Kernel launches issued by this solver since creation (instrumentation).  */
int lbman_launch_count(lbman_solver* s, int64_t* launches);

#ifdef __cplusplus
}
#endif
#endif
