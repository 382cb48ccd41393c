// ens_api.cu -- C ABI of the ensemble runner (lbman_ensemble_*): many
// independent boxes with their own size, boundary configuration and physical
// parameters, advanced together by one launch per kernel per time step
// (ens.cuh), replayed from CUDA graphs.  Host code only.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/lbman3d.h"
#include "ens_launch.h"
#include "solver_view.h"
#include "launch.h"
#include "tiles.h"

namespace lbman {
void set_last_error(const char* msg);
int validate_config(const lbman_config& c);
void build_sim_params(const lbman_config& c, SimParams& P);
}  // namespace lbman

using namespace lbman;

namespace {

int efail(int code, const char* msg) {
    set_last_error(msg);
    return code;
}

#define E_CUDA(call)                                                                      \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            set_last_error(cudaGetErrorString(e_));                                       \
            return e_ == cudaErrorMemoryAllocation ? LBMAN_ERR_NOMEM : LBMAN_ERR_CUDA;    \
        }                                                                                 \
    } while (0)

struct PrecOps {
    decltype(&ens_qstep_f64) qstep;
    decltype(&ens_lbm_f64) lbm;
    decltype(&ens_prepare_f64) prepare;
    decltype(&ens_blocks_per_sm_f64) blocks_per_sm;
    decltype(&launch_seeded_init_f64) seeded_init;
    decltype(&launch_feq_init_f64) feq_init;
    decltype(&launch_real_in_f64) real_in;
    decltype(&launch_real_out_f64) real_out;
    decltype(&launch_pop_in_f64) pop_in;
    decltype(&launch_pop_out_f64) pop_out;
    decltype(&launch_stream_only_f64) stream_only;
    decltype(&qforce_smem_f64) qforce_smem;
    decltype(&qforce_threads_f64) qforce_threads;
};
#define ENS_OPS(S)                                                                                          \
    PrecOps {                                                                                               \
        ens_qstep_##S, ens_lbm_##S, ens_prepare_##S, ens_blocks_per_sm_##S, launch_seeded_init_##S,         \
            launch_feq_init_##S, launch_real_in_##S, launch_real_out_##S, launch_pop_in_##S,                \
            launch_pop_out_##S, launch_stream_only_##S, qforce_smem_##S, qforce_threads_##S                 \
    }
const PrecOps kEnsOps[3] = {ENS_OPS(f64), ENS_OPS(f32), ENS_OPS(f16)};


}  // namespace

struct lbman_ensemble {
    int n = 0, prec = LBMAN_FP32, device = 0, num_sms = 148;
    bool upwind = false;
    size_t rbytes = 4, sbytes = 4;
    std::vector<EnsBox> host;             // per-box descriptors (host copy)
    EnsBox* dboxes = nullptr;
    std::vector<void*> allocs;            // per-box field buffers
    double* staging = nullptr;            // largest box's V doubles
    int64_t maxV = 0, cells = 0;
    // launch shape, work lists
    int kernels = LBMAN_KERNELS_SPLIT, tcx = 32, tcy = 6, zc_target = 0;
    EnsQWork* qwork = nullptr;
    EnsLbmWork* lwork = nullptr;
    int nq = 0, nl = 0, qgrid = 0, lgrid = 0;
    int par = 0;
    bool uploaded = false, f_post = false;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    cudaGraphExec_t graph = nullptr;
    int graph_steps = 0, graph_par = -1;
    int64_t steps = 0, launches = 0;
    const PrecOps& ops() const { return kEnsOps[prec]; }
};

namespace {

void drop_graph(lbman_ensemble* e) {
    if (e->graph) cudaGraphExecDestroy(e->graph);
    e->graph = nullptr;
    e->graph_steps = 0;
    e->graph_par = -1;
}

// Work lists for the current tile: one Q item per z-marching block of each
// box, one LBM item per 256-cell block of each box.
int build_work(lbman_ensemble* e) {
    std::vector<EnsQWork> q;
    std::vector<EnsLbmWork> l;
    for (int b = 0; b < e->n; ++b) {
        EnsBox& B = e->host[b];
        const int gx = (B.P.nx + e->tcx - 1) / e->tcx, gy = (B.P.ny + e->tcy - 1) / e->tcy;
        int zc = e->zc_target > 0 ? std::min(e->zc_target, B.P.nz) : B.P.nz;
        if (e->zc_target <= 0) {  // enough z chunks that big boxes split across SMs
            const long cols = (long)gx * gy;
            long nch = std::max(1L, std::min((long)std::max(1, B.P.nz / 8), (long)(e->num_sms * 2 + cols - 1) / cols));
            zc = (int)((B.P.nz + nch - 1) / nch);
        }
        B.zc = zc;
        const int gz = (B.P.nz + zc - 1) / zc;
        for (int z = 0; z < gz; ++z)
            for (int y = 0; y < gy; ++y)
                for (int x = 0; x < gx; ++x) q.push_back({b, x, y, z});
        const int lb = (int)((B.P.V + 255) / 256);
        for (int k = 0; k < lb; ++k) l.push_back({b, k});
    }
    // largest boxes first: long items start early, short ones fill the tail
    std::stable_sort(q.begin(), q.end(), [&](const EnsQWork& a, const EnsQWork& c) {
        return e->host[a.box].P.V > e->host[c.box].P.V;
    });
    cudaFree(e->qwork);
    cudaFree(e->lwork);
    e->qwork = nullptr;
    e->lwork = nullptr;
    E_CUDA(cudaMalloc(&e->qwork, q.size() * sizeof(EnsQWork)));
    E_CUDA(cudaMalloc(&e->lwork, l.size() * sizeof(EnsLbmWork)));
    // On the ensemble's (non-blocking) stream and waited for: a plain
    // cudaMemcpy from pageable memory may return before its DMA lands, and
    // the legacy stream does not order the kernels queued on this one.
    E_CUDA(cudaMemcpyAsync(e->qwork, q.data(), q.size() * sizeof(EnsQWork), cudaMemcpyHostToDevice, e->stream));
    E_CUDA(cudaMemcpyAsync(e->lwork, l.data(), l.size() * sizeof(EnsLbmWork), cudaMemcpyHostToDevice, e->stream));
    E_CUDA(cudaMemcpyAsync(e->dboxes, e->host.data(), e->n * sizeof(EnsBox), cudaMemcpyHostToDevice, e->stream));
    E_CUDA(cudaStreamSynchronize(e->stream));
    e->nq = (int)q.size();
    e->nl = (int)l.size();
    const int bps = std::max(1, e->ops().blocks_per_sm(e->tcx, e->tcy, e->kernels == LBMAN_KERNELS_FUSED));
    e->qgrid = std::max(1, std::min(e->nq, bps * e->num_sms));
    e->lgrid = std::max(1, std::min(e->nl, 8 * e->num_sms));
    drop_graph(e);
    return LBMAN_OK;
}

// One time step of every box (no graph).
int ens_step_once(lbman_ensemble* e, bool last) {
    const int first = e->f_post ? 0 : 1;
    EnsQLaunch L{e->dboxes, e->qwork, e->nq, e->tcx, e->tcy, e->kernels == LBMAN_KERNELS_FUSED, e->upwind,
                 e->par, first, last ? 1 : 0, e->qgrid};
    cudaError_t err = e->ops().qstep(L, e->stream);
    ++e->launches;
    if (err == cudaSuccess && e->kernels == LBMAN_KERNELS_SPLIT) {
        err = e->ops().lbm(e->dboxes, e->lwork, e->nl, e->par, first, last ? 1 : 0, e->lgrid, e->stream);
        ++e->launches;
    }
    if (err != cudaSuccess) return efail(LBMAN_ERR_CUDA, cudaGetErrorString(err));
    e->par ^= 1;
    e->f_post = true;
    ++e->steps;
    return LBMAN_OK;
}

// Graph of k steps starting at parity e->par (after the first step).
int ens_build_graph(lbman_ensemble* e, int k) {
    drop_graph(e);
    const int par0 = e->par;
    const int64_t steps0 = e->steps, launches0 = e->launches;
    cudaGraph_t g = nullptr;
    E_CUDA(cudaStreamBeginCapture(e->stream, cudaStreamCaptureModeThreadLocal));
    int st = LBMAN_OK;
    for (int i = 0; i < k && st == LBMAN_OK; ++i) st = ens_step_once(e, false);
    cudaError_t ce = cudaStreamEndCapture(e->stream, &g);
    e->par = par0;
    e->steps = steps0;
    e->launches = launches0;
    if (st != LBMAN_OK) {
        if (g) cudaGraphDestroy(g);
        return st;
    }
    if (ce != cudaSuccess) return efail(LBMAN_ERR_CUDA, cudaGetErrorString(ce));
    cudaError_t ie = cudaGraphInstantiate(&e->graph, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) return efail(LBMAN_ERR_CUDA, cudaGetErrorString(ie));
    e->graph_steps = k;
    e->graph_par = par0;
    return LBMAN_OK;
}

}  // namespace

namespace lbman {
int ensemble_box_view(lbman_ensemble* e, int box, SolverView* v) {
    if (!e || !v || box < 0 || box >= e->n) return efail(LBMAN_ERR_ARG, "bad ensemble box");
    const EnsBox& B = e->host[box];
    v->prec = e->prec;
    v->nx = B.P.nx;
    v->ny = B.P.ny;
    v->nz = B.P.nz;
    v->V = B.P.V;
    v->rho = B.rho;
    // the velocity lives in u[0] (split) or in the buffer of the current parity (fused)
    v->u = e->kernels == LBMAN_KERNELS_FUSED ? B.u[e->par] : B.u[0];
    v->q = B.q[e->par];
    v->stream = e->stream;
    v->uploaded = e->uploaded;
    return LBMAN_OK;
}
}  // namespace lbman

extern "C" {

int lbman_ensemble_create(const lbman_config* cfgs, int nboxes, lbman_ensemble** out) {
    if (!cfgs || nboxes < 1 || !out) return efail(LBMAN_ERR_ARG, "need at least one box configuration");
    *out = nullptr;
    for (int b = 0; b < nboxes; ++b)
        if (int st = validate_config(cfgs[b])) return st;
    for (int b = 1; b < nboxes; ++b) {
        if (cfgs[b].precision != cfgs[0].precision || cfgs[b].advection != cfgs[0].advection ||
            cfgs[b].device != cfgs[0].device)
            return efail(LBMAN_ERR_ARG, "all boxes of an ensemble share precision, advection and device");
    }
    lbman_ensemble* e = new lbman_ensemble();
    auto bail = [&](int code) {
        lbman_ensemble_destroy(e);
        return code;
    };
    e->n = nboxes;
    e->prec = cfgs[0].precision;
    e->device = cfgs[0].device;
    e->upwind = cfgs[0].advection == LBMAN_UPWIND;
    e->rbytes = e->prec == LBMAN_FP64 ? 8 : 4;
    e->sbytes = e->prec == LBMAN_FP64 ? 8 : (e->prec == LBMAN_FP32 ? 4 : 2);
    if (cudaSetDevice(e->device) != cudaSuccess) return bail(efail(LBMAN_ERR_CUDA, "cudaSetDevice failed"));
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, e->device) != cudaSuccess)
        return bail(efail(LBMAN_ERR_CUDA, "cudaGetDeviceProperties failed"));
    e->num_sms = prop.multiProcessorCount;
    if (e->ops().prepare(prop.sharedMemPerBlockOptin) != cudaSuccess)
        return bail(efail(LBMAN_ERR_CUDA, "cudaFuncSetAttribute failed"));
    e->kernels = cfgs[0].kernels == LBMAN_KERNELS_FUSED ? LBMAN_KERNELS_FUSED : LBMAN_KERNELS_SPLIT;
    if (cfgs[0].tile_x > 0 && cfgs[0].tile_y > 0) {
        e->tcx = cfgs[0].tile_x;
        e->tcy = cfgs[0].tile_y;
    } else if (e->prec == LBMAN_FP64) {
        e->tcx = 30;
        e->tcy = 6;
    }
    if (e->ops().qforce_smem(QTile{e->tcx, e->tcy, 1}) == 0)
        return bail(efail(LBMAN_ERR_ARG, "tile is not compiled for this precision"));
    e->zc_target = cfgs[0].zchunk;
    e->host.resize(nboxes);
    for (int b = 0; b < nboxes; ++b) {
        EnsBox& B = e->host[b];
        std::memset(&B, 0, sizeof(B));
        build_sim_params(cfgs[b], B.P);
        B.dnx = make_fastdiv((uint32_t)B.P.nx);
        B.dnxy = make_fastdiv((uint32_t)B.P.nxy);
        const int64_t V = B.P.V;
        e->maxV = std::max(e->maxV, V);
        e->cells += V;
        void** slots[8] = {&B.q[0], &B.q[1], &B.u[0], &B.u[1], &B.f[0], &B.f[1], &B.rho, &B.F};
        const size_t sizes[8] = {5 * V * e->rbytes, 5 * V * e->rbytes, 3 * V * e->rbytes, 3 * V * e->rbytes,
                                 15 * V * e->sbytes, 15 * V * e->sbytes, V * e->rbytes, 3 * V * e->rbytes};
        for (int k = 0; k < 8; ++k) {
            if (cudaMalloc(slots[k], sizes[k]) != cudaSuccess)
                return bail(efail(LBMAN_ERR_NOMEM, "cudaMalloc of an ensemble box failed"));
            e->allocs.push_back(*slots[k]);
        }
    }
    if (cudaMalloc(&e->staging, e->maxV * sizeof(double)) != cudaSuccess ||
        cudaMalloc(&e->dboxes, nboxes * sizeof(EnsBox)) != cudaSuccess)
        return bail(efail(LBMAN_ERR_NOMEM, "cudaMalloc failed"));
    if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess)
        return bail(efail(LBMAN_ERR_CUDA, "cudaStreamCreate failed"));
    e->own_stream = true;
    if (int st = build_work(e)) return bail(st);
    *out = e;
    return LBMAN_OK;
}

int lbman_ensemble_destroy(lbman_ensemble* e) {
    if (!e) return LBMAN_OK;
    cudaSetDevice(e->device);
    if (e->stream) cudaStreamSynchronize(e->stream);
    drop_graph(e);
    for (void* p : e->allocs) cudaFree(p);
    cudaFree(e->staging);
    cudaFree(e->dboxes);
    cudaFree(e->qwork);
    cudaFree(e->lwork);
    if (e->own_stream && e->stream) cudaStreamDestroy(e->stream);
    delete e;
    return LBMAN_OK;
}

int lbman_ensemble_set_stream(lbman_ensemble* e, void* stream) {
    if (!e) return efail(LBMAN_ERR_ARG, "null ensemble");
    E_CUDA(cudaStreamSynchronize(e->stream));
    if (e->own_stream) cudaStreamDestroy(e->stream);
    e->stream = (cudaStream_t)stream;
    e->own_stream = false;
    drop_graph(e);
    return LBMAN_OK;
}

int lbman_ensemble_init_seeded(lbman_ensemble* e, uint64_t seed, double sigma) {
    if (!e) return efail(LBMAN_ERR_ARG, "null ensemble");
    std::vector<uint64_t> seeds((size_t)e->n);
    for (int b = 0; b < e->n; ++b) seeds[(size_t)b] = seed + (uint64_t)b;
    return lbman_ensemble_init_seeded_each(e, seeds.data(), sigma);
}

int lbman_ensemble_init_seeded_each(lbman_ensemble* e, const uint64_t* seeds, double sigma) {
    if (!e || !seeds) return efail(LBMAN_ERR_ARG, "null argument");
    E_CUDA(cudaSetDevice(e->device));
    e->par = 0;
    for (int b = 0; b < e->n; ++b) {
        EnsBox& B = e->host[b];
        const SimParams& P = B.P;
        // ordered root of the bulk Landau-de Gennes field (src/model.h:39-41)
        const double S0 = (-P.B + std::sqrt(P.B * P.B - 24.0 * P.A * P.C)) / (4.0 * P.C);
        if (e->ops().seeded_init(P, seeds[b], S0, sigma, B.rho, B.u[0], B.q[0], B.F, e->stream) != cudaSuccess ||
            e->ops().feq_init(P, B.rho, B.u[0], B.f[0], e->stream) != cudaSuccess)
            return efail(LBMAN_ERR_CUDA, "seeded initialisation failed");
        E_CUDA(cudaMemcpyAsync(B.u[1], B.u[0], 3 * P.V * e->rbytes, cudaMemcpyDeviceToDevice, e->stream));
        e->launches += 2;
    }
    E_CUDA(cudaStreamSynchronize(e->stream));
    e->uploaded = true;
    e->f_post = false;
    e->steps = 0;
    drop_graph(e);
    return LBMAN_OK;
}

int lbman_ensemble_upload(lbman_ensemble* e, int box, const double* rho, const double* u3, const double* q5) {
    if (!e || box < 0 || box >= e->n || !rho || !u3 || !q5) return efail(LBMAN_ERR_ARG, "bad arguments");
    if (e->uploaded && e->f_post) return efail(LBMAN_ERR_STATE, "boxes are uploaded before the first step");
    E_CUDA(cudaSetDevice(e->device));
    EnsBox& B = e->host[box];
    const SimParams& P = B.P;
    const int64_t V = P.V;
    auto in = [&](const double* src, void* dst, int64_t n) -> int {
        for (int64_t off = 0; off < n; off += V) {
            void* d = (char*)dst + off * e->rbytes;
            if (e->prec == LBMAN_FP64) {
                E_CUDA(cudaMemcpyAsync(d, src + off, V * 8, cudaMemcpyHostToDevice, e->stream));
            } else {
                E_CUDA(cudaMemcpyAsync(e->staging, src + off, V * 8, cudaMemcpyHostToDevice, e->stream));
                if (e->ops().real_in(e->staging, d, V, e->stream) != cudaSuccess)
                    return efail(LBMAN_ERR_CUDA, "conversion failed");
            }
        }
        return LBMAN_OK;
    };
    e->par = 0;
    if (int st = in(rho, B.rho, V)) return st;
    if (int st = in(u3, B.u[0], 3 * V)) return st;
    if (int st = in(q5, B.q[0], 5 * V)) return st;
    E_CUDA(cudaMemcpyAsync(B.u[1], B.u[0], 3 * V * e->rbytes, cudaMemcpyDeviceToDevice, e->stream));
    E_CUDA(cudaMemsetAsync(B.F, 0, 3 * V * e->rbytes, e->stream));
    if (e->ops().feq_init(P, B.rho, B.u[0], B.f[0], e->stream) != cudaSuccess)
        return efail(LBMAN_ERR_CUDA, "f_eq initialisation failed");
    E_CUDA(cudaStreamSynchronize(e->stream));
    e->uploaded = true;
    e->f_post = false;
    e->steps = 0;
    drop_graph(e);
    return LBMAN_OK;
}

int lbman_ensemble_download(lbman_ensemble* e, int box, double* rho, double* u3, double* q5, double* f15) {
    if (!e || box < 0 || box >= e->n) return efail(LBMAN_ERR_ARG, "bad arguments");
    if (!e->uploaded) return efail(LBMAN_ERR_STATE, "download before initialisation");
    E_CUDA(cudaSetDevice(e->device));
    const EnsBox& B = e->host[box];
    const SimParams& P = B.P;
    const int64_t V = P.V;
    const int p = e->par;
    auto out = [&](const void* src, double* dst, int64_t n) -> int {
        for (int64_t off = 0; off < n; off += V) {
            const void* s = (const char*)src + off * e->rbytes;
            if (e->prec == LBMAN_FP64) {
                E_CUDA(cudaMemcpyAsync(dst + off, s, V * 8, cudaMemcpyDeviceToHost, e->stream));
            } else {
                if (e->ops().real_out(s, e->staging, V, e->stream) != cudaSuccess)
                    return efail(LBMAN_ERR_CUDA, "conversion failed");
                E_CUDA(cudaMemcpyAsync(dst + off, e->staging, V * 8, cudaMemcpyDeviceToHost, e->stream));
            }
            E_CUDA(cudaStreamSynchronize(e->stream));
        }
        return LBMAN_OK;
    };
    // the velocity lives in u[0] (split) or in the buffer of the current parity (fused)
    const void* u = e->kernels == LBMAN_KERNELS_FUSED ? B.u[p] : B.u[0];
    if (rho) if (int st = out(B.rho, rho, V)) return st;
    if (u3) if (int st = out(u, u3, 3 * V)) return st;
    if (q5) if (int st = out(B.q[p], q5, 5 * V)) return st;
    if (f15) {
        const void* src = B.f[p];
        if (e->f_post) {
            if (e->ops().stream_only(P, B.f[p], B.f[1 - p], B.rho, e->stream) != cudaSuccess)
                return efail(LBMAN_ERR_CUDA, "stream failed");
            src = B.f[1 - p];
        }
        for (int j = 0; j < 15; ++j) {
            if (e->prec == LBMAN_FP64) {
                E_CUDA(cudaMemcpyAsync(f15 + j * V, (const char*)src + j * V * 8, V * 8, cudaMemcpyDeviceToHost, e->stream));
            } else {
                if (e->ops().pop_out(P, src, e->staging, j, e->stream) != cudaSuccess)
                    return efail(LBMAN_ERR_CUDA, "conversion failed");
                E_CUDA(cudaMemcpyAsync(f15 + j * V, e->staging, V * 8, cudaMemcpyDeviceToHost, e->stream));
            }
            E_CUDA(cudaStreamSynchronize(e->stream));
        }
    }
    E_CUDA(cudaStreamSynchronize(e->stream));
    return LBMAN_OK;
}

int lbman_ensemble_step(lbman_ensemble* e, int nsteps) {
    if (!e || nsteps < 0) return efail(LBMAN_ERR_ARG, "bad arguments");
    if (!e->uploaded) return efail(LBMAN_ERR_STATE, "step before initialisation");
    E_CUDA(cudaSetDevice(e->device));
    int done = 0;
    // rho everywhere is refreshed by the final step of each call
    if (!e->f_post && nsteps > 0) {
        if (int st = ens_step_once(e, nsteps == 1)) return st;
        ++done;
    }
    constexpr int kGraphSteps = 20;  // even, so a replay keeps the buffer parity
    while (nsteps - done > kGraphSteps) {
        if (!e->graph || e->graph_par != e->par) {
            if (int st = ens_build_graph(e, kGraphSteps)) return st;
        }
        E_CUDA(cudaGraphLaunch(e->graph, e->stream));
        e->launches += (int64_t)kGraphSteps * (e->kernels == LBMAN_KERNELS_SPLIT ? 2 : 1);
        e->steps += kGraphSteps;
        done += kGraphSteps;
    }
    while (done < nsteps) {
        if (int st = ens_step_once(e, done == nsteps - 1)) return st;
        ++done;
    }
    return LBMAN_OK;
}

int lbman_ensemble_synchronize(lbman_ensemble* e) {
    if (!e) return efail(LBMAN_ERR_ARG, "null ensemble");
    E_CUDA(cudaStreamSynchronize(e->stream));
    return LBMAN_OK;
}

int lbman_ensemble_set_shape(lbman_ensemble* e, int kernels, int tile_x, int tile_y, int zchunk) {
    if (!e) return efail(LBMAN_ERR_ARG, "null ensemble");
    if (kernels != LBMAN_KERNELS_SPLIT && kernels != LBMAN_KERNELS_FUSED)
        return efail(LBMAN_ERR_ARG, "kernels must be SPLIT or FUSED");
    if (e->ops().qforce_smem(QTile{tile_x, tile_y, 1}) == 0)
        return efail(LBMAN_ERR_ARG, "tile is not compiled for this precision");
    if (e->f_post && kernels != e->kernels) {
        // the split organisation keeps u in u[0]; the fused one ping-pongs
        const int p = e->par;
        for (auto& B : e->host) {
            if (kernels == LBMAN_KERNELS_FUSED && p != 0)
                E_CUDA(cudaMemcpyAsync(B.u[p], B.u[0], 3 * B.P.V * e->rbytes, cudaMemcpyDeviceToDevice, e->stream));
            if (kernels == LBMAN_KERNELS_SPLIT && p != 0)
                E_CUDA(cudaMemcpyAsync(B.u[0], B.u[p], 3 * B.P.V * e->rbytes, cudaMemcpyDeviceToDevice, e->stream));
        }
        E_CUDA(cudaStreamSynchronize(e->stream));
    }
    e->kernels = kernels;
    e->tcx = tile_x;
    e->tcy = tile_y;
    e->zc_target = zchunk;
    return build_work(e);
}

int lbman_ensemble_get_shape(lbman_ensemble* e, lbman_shape* out) {
    if (!e || !out) return efail(LBMAN_ERR_ARG, "null argument");
    out->kernels = e->kernels;
    out->tile_x = e->tcx;
    out->tile_y = e->tcy;
    out->zchunk = e->zc_target;
    out->threads = e->ops().qforce_threads(QTile{e->tcx, e->tcy, 1});
    out->ms_per_step = 0.0;
    return LBMAN_OK;
}

int lbman_ensemble_autotune(lbman_ensemble* e, int steps_per_trial, lbman_shape* best, int* ntrials) {
    if (!e || !best || steps_per_trial < 1) return efail(LBMAN_ERR_ARG, "bad arguments");
    if (!e->uploaded) return efail(LBMAN_ERR_STATE, "autotune needs an initialised ensemble");
    E_CUDA(cudaSetDevice(e->device));
    // Snapshot every box so the trials leave no trace.
    std::vector<void*> snap;
    auto bytes_of = [&](const EnsBox& B, int k) -> size_t {
        const int64_t V = B.P.V;
        const size_t s[8] = {5 * V * e->rbytes, 5 * V * e->rbytes, 3 * V * e->rbytes, 3 * V * e->rbytes,
                             15 * V * e->sbytes, 15 * V * e->sbytes, V * e->rbytes, 3 * V * e->rbytes};
        return s[k];
    };
    auto ptr_of = [&](EnsBox& B, int k) -> void* {
        void* p[8] = {B.q[0], B.q[1], B.u[0], B.u[1], B.f[0], B.f[1], B.rho, B.F};
        return p[k];
    };
    for (auto& B : e->host)
        for (int k = 0; k < 8; ++k) {
            void* p = nullptr;
            if (cudaMalloc(&p, bytes_of(B, k)) != cudaSuccess) {
                for (void* q : snap) cudaFree(q);
                return efail(LBMAN_ERR_NOMEM, "autotune snapshot allocation failed");
            }
            snap.push_back(p);
            E_CUDA(cudaMemcpyAsync(p, ptr_of(B, k), bytes_of(B, k), cudaMemcpyDeviceToDevice, e->stream));
        }
    const int par0 = e->par, kern0 = e->kernels, tx0 = e->tcx, ty0 = e->tcy, zc0 = e->zc_target;
    const bool fpost0 = e->f_post;
    const int64_t steps0 = e->steps;
    cudaEvent_t a = nullptr, b = nullptr;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    lbman_shape win{kern0, tx0, ty0, zc0, 0, 1e30};
    int count = 0, status = LBMAN_OK;
    for (int k : {LBMAN_KERNELS_SPLIT, LBMAN_KERNELS_FUSED}) {
        for (const auto& t : kTileList) {
            if (e->ops().qforce_smem(QTile{t[0], t[1], 1}) == 0) continue;
            for (int zc : {0, 16, 48}) {
                if ((status = lbman_ensemble_set_shape(e, k, t[0], t[1], zc)) != LBMAN_OK) break;
                if ((status = ens_step_once(e, false)) != LBMAN_OK) break;
                cudaEventRecord(a, e->stream);
                for (int n = 0; n < steps_per_trial && status == LBMAN_OK; ++n) status = ens_step_once(e, false);
                cudaEventRecord(b, e->stream);
                if (status != LBMAN_OK || cudaEventSynchronize(b) != cudaSuccess) {
                    if (status == LBMAN_OK) status = efail(LBMAN_ERR_CUDA, "autotune trial failed");
                    break;
                }
                float ms = 0.f;
                cudaEventElapsedTime(&ms, a, b);
                ++count;
                if (ms / steps_per_trial < win.ms_per_step) win = {k, t[0], t[1], zc, 0, ms / steps_per_trial};
            }
            if (status != LBMAN_OK) break;
        }
        if (status != LBMAN_OK) break;
    }
    // restore: fields, parity and the velocity organisation of the original shape
    e->kernels = kern0;
    int i = 0;
    for (auto& B : e->host)
        for (int k = 0; k < 8; ++k, ++i)
            cudaMemcpyAsync(ptr_of(B, k), snap[i], bytes_of(B, k), cudaMemcpyDeviceToDevice, e->stream);
    cudaStreamSynchronize(e->stream);
    for (void* p : snap) cudaFree(p);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    e->par = par0;
    e->f_post = fpost0;
    e->steps = steps0;
    if (status != LBMAN_OK) {
        lbman_ensemble_set_shape(e, kern0, tx0, ty0, zc0);
        return status;
    }
    if (int st = lbman_ensemble_set_shape(e, win.kernels, win.tile_x, win.tile_y, win.zchunk)) return st;
    *best = win;
    best->threads = e->ops().qforce_threads(QTile{win.tile_x, win.tile_y, 1});
    if (ntrials) *ntrials = count;
    return LBMAN_OK;
}

int lbman_ensemble_info(lbman_ensemble* e, int64_t* cells, int64_t* steps, int64_t* launches) {
    if (!e) return efail(LBMAN_ERR_ARG, "null ensemble");
    if (cells) *cells = e->cells;
    if (steps) *steps = e->steps;
    if (launches) *launches = e->launches;
    return LBMAN_OK;
}

}  // extern "C"
