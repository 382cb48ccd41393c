// closure_api.cu -- C ABI of the learned closure (no counterpart in the
// reference).  A coarse FP32 solver on an f-times coarser periodic grid is
// advanced with the plain method, and after every coarse step a 3D CNN
// (closure.cuh) corrects its Q and u.  The CNN sees the state before the
// step; it is trained on box-filtered fine-grid snapshots to predict
// filtered(fine, t + 1 coarse step) - coarse_step(filtered(fine, t)).
//
// Coarse step operator: populations rebuilt as f_eq(rho, u) of the current
// fields, then one solver step (lbman_step) -- the same operator in training
// and in the corrected run.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/lbman3d.h"
#include "closure.cuh"
#include "closure_selftest.cuh"
#include "solver_view.h"

using namespace lbman;

namespace {

// ---- network shape ----------------------------------------------------------
struct LayerDef {
    int cin, cout, real_cin, real_cout;
};
constexpr LayerDef kLayers[4] = {{16, 32, 9, 32}, {32, 32, 32, 32}, {32, 32, 32, 32}, {32, 16, 32, 8}};
constexpr int w_size(int l) { return 27 * kLayers[l].cin * kLayers[l].cout; }
constexpr int w_off(int l) { return l == 0 ? 0 : w_off(l - 1) + w_size(l - 1) + kLayers[l - 1].cout; }
constexpr int b_off(int l) { return w_off(l) + w_size(l); }
constexpr int kNParams = b_off(3) + kLayers[3].cout;

float bf16_round(float x) {
    uint32_t u;
    std::memcpy(&u, &x, 4);
    const uint32_t lsb = (u >> 16) & 1u;
    u = (u + 0x7FFFu + lsb) & 0xFFFF0000u;
    float y;
    std::memcpy(&y, &u, 4);
    return y;
}

char g_msg[512];
int failc(int code, const char* msg) {
    std::snprintf(g_msg, sizeof(g_msg), "%s", msg);
    set_last_error(g_msg);
    return code;
}
int cuda_fail(cudaError_t e, const char* what) {
    std::snprintf(g_msg, sizeof(g_msg), "%s: %s", what, cudaGetErrorString(e));
    set_last_error(g_msg);
    return e == cudaErrorMemoryAllocation ? LBMAN_ERR_NOMEM : LBMAN_ERR_CUDA;
}
#define CL_CUDA(x)                                \
    do {                                          \
        cudaError_t e_ = (x);                     \
        if (e_ != cudaSuccess) return cuda_fail(e_, #x); \
    } while (0)
#define CL_TRY(x)                         \
    do {                                  \
        int s_ = (x);                     \
        if (s_ != LBMAN_OK) return s_;    \
    } while (0)

template <auto Kern>
int resident(int threads, size_t smem) {
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, Kern, threads, smem) != cudaSuccess || n < 1) {
        cudaGetLastError();
        n = 1;
    }
    return n;
}

// Resident blocks per SM of a kernel at this launch shape, from the device's
// shared memory per SM (1 KB reserved per block), the kernel's registers and
// static shared memory, and the thread limit.
template <auto Kern>
int fit_blocks(int device, int threads, size_t dyn_smem) {
    int smem_sm = 0, regs_sm = 0, threads_sm = 0;
    cudaFuncAttributes fa{};
    if (cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&regs_sm, cudaDevAttrMaxRegistersPerMultiprocessor, device) != cudaSuccess ||
        cudaDeviceGetAttribute(&threads_sm, cudaDevAttrMaxThreadsPerMultiProcessor, device) != cudaSuccess ||
        cudaFuncGetAttributes(&fa, Kern) != cudaSuccess) {
        cudaGetLastError();
        return 1;
    }
    const size_t per_block = dyn_smem + fa.sharedSizeBytes + 1024;
    int n = (int)((size_t)smem_sm / per_block);
    n = std::min(n, regs_sm / std::max(1, fa.numRegs * threads));
    n = std::min(n, threads_sm / threads);
    return std::max(1, n);
}

}  // namespace

struct lbman_closure {
    int device = 0, nx = 0, ny = 0, nz = 0, num_sms = 148;
    int64_t V = 0;
    cudaStream_t stream = nullptr;
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr, *mask = nullptr;
    int64_t adam_t = 0;
    __nv_bfloat16* fimg[4] = {nullptr, nullptr, nullptr, nullptr};
    __nv_bfloat16* bimg[4] = {nullptr, nullptr, nullptr, nullptr};
    __nv_bfloat16 *act0 = nullptr, *gout = nullptr;
    __nv_bfloat16* act[3] = {nullptr, nullptr, nullptr};
    __nv_bfloat16* pre[3] = {nullptr, nullptr, nullptr};
    __nv_bfloat16* gbuf[2] = {nullptr, nullptr};
    float* out = nullptr;
    float* wpart = nullptr;
    float* bpart = nullptr;
    double* lpart = nullptr;
    double* loss_hist = nullptr;
    int loss_cap = 0;
    float* scales = nullptr;  // shift[9] inv_scale[9] out_scale[8] inv_out_scale[8]
    float h_shift[9], h_scale[9], h_out[8];
    int* err = nullptr;
    uint32_t wait_limit = lbman::tc::kWaitLimit;  // polls of a pipeline wait before it gives up
    int Gw = 148, Gb = 296;
    std::vector<float*> snaps;          // filtered fine states [9V] (rho, u, Q), in recording order
    std::vector<int> traj;              // trajectory id of each snapshot
    std::vector<float*> targets;        // training pairs: target [8V] ...
    std::vector<const float*> pair_in;  // ... and the input state it corrects
    std::vector<float*> rollout_in;     // inputs of the rollout pairs (corrected-run states), owned
    int cur_traj = -1;
    float train_noise = 0.0f;  // std of N(0,1) noise on the normalised inputs in training
    float gain = 1.0f;         // correction multiplier in lbman_closure_step
};

namespace {

template <int CIN, int COUT, int MODE>
int run_conv(lbman_closure* c, cudaStream_t st, const __nv_bfloat16* in, const __nv_bfloat16* img,
             const float* bias, const __nv_bfloat16* pre_below, __nv_bfloat16* out_pre, __nv_bfloat16* out_bf,
             float* out_f) {
    if (cl::dhalo_ok(c->nx, c->ny)) {
        constexpr size_t smem = cl::bimg_bytes(CIN, COUT) + cl::dhalo_bytes(CIN);
        constexpr auto K = cl::conv_dhalo_kernel<CIN, COUT, MODE>;
        CL_CUDA(cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        // all of the unified L1 / shared memory as shared memory: two blocks
        // per SM
        CL_CUDA(cudaFuncSetAttribute(K, cudaFuncAttributePreferredSharedMemoryCarveout, 100));
        // one block per (column, z range): as many z ranges as keep every
        // column's blocks within one wave of resident blocks (counted from
        // the SM's shared memory, registers and threads)
        const int cols = (c->nx / 8) * (c->ny / 16);
        const int slots = fit_blocks<K>(c->device, cl::kZThreads, smem) * c->num_sms;
        const int nch = std::max(1, std::min(c->nz, slots / cols));
        const int zc = (c->nz + nch - 1) / nch;
        const int grid = cols * ((c->nz + zc - 1) / zc);
        const cl::Grid3 gr{c->nx, c->ny, c->nz, c->V};
        K<<<grid, cl::kZThreads, smem, st>>>(gr, zc, in, reinterpret_cast<const uint4*>(img), bias, pre_below,
                                             out_pre, out_bf, out_f, c->err, c->wait_limit);
        CL_CUDA(cudaGetLastError());
        return LBMAN_OK;
    }
    const int halo = cl::halo_ok(c->nx, c->ny) && cl::halo_bytes(c->nx, CIN) <= 96 * 1024 ? 1 : 0;
    const size_t smem =
        cl::bimg_bytes(CIN, COUT) + cl::kStages * (CIN / 16) * 4096 + (halo ? cl::halo_bytes(c->nx, CIN) : 0);
    constexpr auto K = cl::conv_kernel<CIN, COUT, MODE>;
    CL_CUDA(cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int64_t tiles = (c->V + cl::kTileM - 1) / cl::kTileM;
    const int grid = (int)std::min<int64_t>(tiles, (int64_t)resident<K>(cl::kThreads, smem) * c->num_sms);
    const cl::Grid3 gr{c->nx, c->ny, c->nz, c->V};
    K<<<grid, cl::kThreads, smem, st>>>(gr, in, reinterpret_cast<const uint4*>(img), bias, pre_below, out_pre, out_bf,
                                        out_f, halo, c->err, c->wait_limit);
    CL_CUDA(cudaGetLastError());
    return LBMAN_OK;
}

template <int CIN, int COUT>
int run_wgrad(lbman_closure* c, cudaStream_t st, const __nv_bfloat16* a, const __nv_bfloat16* gr, int layer) {
    const cl::Grid3 g3{c->nx, c->ny, c->nz, c->V};
    if (cl::dhalo_ok(c->nx, c->ny)) {
        using WH = cl::WGradHalo<CIN, COUT>;
        constexpr auto K = cl::wgrad_dhalo_kernel<CIN, COUT>;
        CL_CUDA(cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, WH::SMEM));
        K<<<c->Gw, cl::kThreads, WH::SMEM, st>>>(g3, a, gr, c->wpart, c->err, c->wait_limit);
    } else {
        using WS = cl::WGradShape<CIN, COUT>;
        constexpr auto K = cl::wgrad_kernel<CIN, COUT>;
        CL_CUDA(cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, WS::SMEM));
        K<<<c->Gw, cl::kThreads, WS::SMEM, st>>>(g3, a, gr, c->wpart, c->err, c->wait_limit);
    }
    CL_CUDA(cudaGetLastError());
    const int n = 27 * CIN * COUT;
    cl::sum_partials_kernel<<<(n + 31) / 32, cl::kFoldThreads, 0, st>>>(c->wpart, c->Gw, n, c->g + w_off(layer));
    CL_CUDA(cudaGetLastError());
    return LBMAN_OK;
}

template <int C>
int run_bias_grad(lbman_closure* c, cudaStream_t st, const __nv_bfloat16* gr, int layer) {
    cl::bias_grad_kernel<C><<<c->Gb, cl::kThreads, 0, st>>>(gr, c->V, c->bpart);
    CL_CUDA(cudaGetLastError());
    cl::sum_partials_kernel<<<(C + 31) / 32, cl::kFoldThreads, 0, st>>>(c->bpart, c->Gb, C, c->g + b_off(layer));
    CL_CUDA(cudaGetLastError());
    return LBMAN_OK;
}

int pack(lbman_closure* c, cudaStream_t st) {
    cl::pack_kernel<16, 32><<<64, 256, 0, st>>>(c->p + w_off(0), c->fimg[0], nullptr);
    cl::pack_kernel<32, 32><<<64, 256, 0, st>>>(c->p + w_off(1), c->fimg[1], c->bimg[1]);
    cl::pack_kernel<32, 32><<<64, 256, 0, st>>>(c->p + w_off(2), c->fimg[2], c->bimg[2]);
    cl::pack_kernel<32, 16><<<64, 256, 0, st>>>(c->p + w_off(3), c->fimg[3], c->bimg[3]);
    CL_CUDA(cudaGetLastError());
    return LBMAN_OK;
}

int upload_scales(lbman_closure* c) {
    float h[34];
    for (int j = 0; j < 9; ++j) {
        h[j] = c->h_shift[j];
        h[9 + j] = 1.0f / c->h_scale[j];
    }
    for (int j = 0; j < 8; ++j) {
        h[18 + j] = c->h_out[j];
        h[26 + j] = 1.0f / c->h_out[j];
    }
    CL_CUDA(cudaMemcpyAsync(c->scales, h, sizeof(h), cudaMemcpyHostToDevice, c->stream));
    CL_CUDA(cudaStreamSynchronize(c->stream));
    return LBMAN_OK;
}

int features(lbman_closure* c, cudaStream_t st, const float* rho, const float* u3, const float* q5,
             float noise_std = 0.0f, uint64_t noise_key = 0) {
    cl::features_kernel<<<c->Gb, 256, 0, st>>>(rho, u3, q5, c->V, c->scales, c->scales + 9, c->act0, noise_std,
                                                noise_key);
    CL_CUDA(cudaGetLastError());
    return LBMAN_OK;
}

int forward(lbman_closure* c, cudaStream_t st) {
    CL_TRY((run_conv<16, 32, cl::kFwdHidden>(c, st, c->act0, c->fimg[0], c->p + b_off(0), nullptr, c->pre[0],
                                             c->act[0], nullptr)));
    CL_TRY((run_conv<32, 32, cl::kFwdHidden>(c, st, c->act[0], c->fimg[1], c->p + b_off(1), nullptr, c->pre[1],
                                             c->act[1], nullptr)));
    CL_TRY((run_conv<32, 32, cl::kFwdHidden>(c, st, c->act[1], c->fimg[2], c->p + b_off(2), nullptr, c->pre[2],
                                             c->act[2], nullptr)));
    CL_TRY((run_conv<32, 16, cl::kFwdLast>(c, st, c->act[2], c->fimg[3], c->p + b_off(3), nullptr, nullptr, nullptr,
                                           c->out)));
    return LBMAN_OK;
}

// Loss gradient gout must be filled; fills c->g.
int backward(lbman_closure* c, cudaStream_t st) {
    CL_TRY((run_wgrad<32, 16>(c, st, c->act[2], c->gout, 3)));
    CL_TRY(run_bias_grad<16>(c, st, c->gout, 3));
    CL_TRY((run_conv<16, 32, cl::kBwdData>(c, st, c->gout, c->bimg[3], nullptr, c->pre[2], nullptr, c->gbuf[0],
                                           nullptr)));
    CL_TRY((run_wgrad<32, 32>(c, st, c->act[1], c->gbuf[0], 2)));
    CL_TRY(run_bias_grad<32>(c, st, c->gbuf[0], 2));
    CL_TRY((run_conv<32, 32, cl::kBwdData>(c, st, c->gbuf[0], c->bimg[2], nullptr, c->pre[1], nullptr, c->gbuf[1],
                                           nullptr)));
    CL_TRY((run_wgrad<32, 32>(c, st, c->act[0], c->gbuf[1], 1)));
    CL_TRY(run_bias_grad<32>(c, st, c->gbuf[1], 1));
    CL_TRY((run_conv<32, 32, cl::kBwdData>(c, st, c->gbuf[1], c->bimg[1], nullptr, c->pre[0], nullptr, c->gbuf[0],
                                           nullptr)));
    CL_TRY((run_wgrad<16, 32>(c, st, c->act0, c->gbuf[0], 0)));
    CL_TRY(run_bias_grad<32>(c, st, c->gbuf[0], 0));
    return LBMAN_OK;
}

int loss_grad(lbman_closure* c, cudaStream_t st, const float* tgt) {
    cl::loss_kernel<<<c->Gb, cl::kThreads, 0, st>>>(c->out, tgt, c->scales + 26, c->V, c->gout, c->lpart);
    CL_CUDA(cudaGetLastError());
    return LBMAN_OK;
}

__global__ void fold_loss_kernel(const double* partials, int G, double scale, double* dst) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < G; ++i) s += partials[i];
        *dst = s * scale;
    }
}

int check_err(lbman_closure* c) {
    int h = 0;
    CL_CUDA(cudaMemcpy(&h, c->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (h) {
        cudaMemsetAsync(c->err, 0, sizeof(int), c->stream);
        cudaStreamSynchronize(c->stream);
        return failc(LBMAN_ERR_TIMEOUT, "closure: a tensor-core wait timed out");
    }
    return LBMAN_OK;
}

float* coarse_f32(lbman_closure* c, lbman_solver* s, SolverView* v) {
    if (solver_view(s, v) != LBMAN_OK) return nullptr;
    if (v->prec == LBMAN_FP64 || v->nx != c->nx || v->ny != c->ny || v->nz != c->nz) return nullptr;
    return static_cast<float*>(v->u);
}

}  // namespace

extern "C" {

int lbman_closure_param_count(void) { return kNParams; }

int lbman_closure_create(int device, int nx, int ny, int nz, uint64_t seed, lbman_closure** out) {
    if (!out || nx < 1 || ny < 1 || nz < 1) return failc(LBMAN_ERR_ARG, "closure: bad arguments");
    *out = nullptr;
    CL_CUDA(cudaSetDevice(device));
    lbman_closure* c = new lbman_closure;
    c->device = device;
    c->nx = nx;
    c->ny = ny;
    c->nz = nz;
    c->V = (int64_t)nx * ny * nz;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) c->num_sms = prop.multiProcessorCount;
    c->Gw = 2 * c->num_sms;  // weight-gradient CTAs (two fit per SM in the staged form)
    c->Gb = 2 * c->num_sms;
    for (int j = 0; j < 9; ++j) {
        c->h_shift[j] = j == 0 ? 1.0f : 0.0f;
        c->h_scale[j] = 1.0f;
    }
    for (int j = 0; j < 8; ++j) c->h_out[j] = 1.0f;
    auto bail = [&](cudaError_t e, const char* w) {
        lbman_closure_destroy(c);
        return cuda_fail(e, w);
    };
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return bail(e, "stream");
    const size_t P = kNParams * sizeof(float);
    const size_t VB = (size_t)c->V * 2;  // one BF16 channel
    struct { void** p; size_t n; } allocs[] = {
        {(void**)&c->p, P}, {(void**)&c->g, P}, {(void**)&c->m, P}, {(void**)&c->v, P}, {(void**)&c->mask, P},
        {(void**)&c->act0, VB * 16}, {(void**)&c->gout, VB * 16},
        {(void**)&c->act[0], VB * 32}, {(void**)&c->act[1], VB * 32}, {(void**)&c->act[2], VB * 32},
        {(void**)&c->pre[0], VB * 32}, {(void**)&c->pre[1], VB * 32}, {(void**)&c->pre[2], VB * 32},
        {(void**)&c->gbuf[0], VB * 32}, {(void**)&c->gbuf[1], VB * 32},
        {(void**)&c->out, (size_t)c->V * 16 * 4},
        {(void**)&c->wpart, (size_t)c->Gw * 27 * 32 * 32 * 4}, {(void**)&c->bpart, (size_t)c->Gb * 32 * 4},
        {(void**)&c->lpart, (size_t)c->Gb * 8}, {(void**)&c->scales, 34 * 4}, {(void**)&c->err, sizeof(int)},
    };
    for (auto& a : allocs) {
        if ((e = cudaMalloc(a.p, a.n)) != cudaSuccess) return bail(e, "closure allocation");
    }
    for (int l = 0; l < 4; ++l) {
        if ((e = cudaMalloc(&c->fimg[l], cl::bimg_bytes(kLayers[l].cin, kLayers[l].cout))) != cudaSuccess)
            return bail(e, "closure allocation");
        if (l > 0 && (e = cudaMalloc(&c->bimg[l], cl::bimg_bytes(kLayers[l].cout, kLayers[l].cin))) != cudaSuccess)
            return bail(e, "closure allocation");
    }
    // He-normal weights (fan-in 27 x real inputs), last layer scaled by 0.1 so
    // the initial correction is small; zero biases; padding entries masked.
    std::vector<float> hp(kNParams, 0.0f), hm(kNParams, 0.0f);
    uint64_t st = seed ^ 0x5851f42d4c957f2dull;
    auto next = [&]() {
        st += 0x9e3779b97f4a7c15ull;
        uint64_t z = st;
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return ((double)((z ^ (z >> 31)) >> 11) + 0.5) * 0x1.0p-53;
    };
    for (int l = 0; l < 4; ++l) {
        const LayerDef& d = kLayers[l];
        const double sd = std::sqrt(2.0 / (27.0 * d.real_cin)) * (l == 3 ? 0.1 : 1.0);
        for (int tap = 0; tap < 27; ++tap)
            for (int ci = 0; ci < d.cin; ++ci)
                for (int co = 0; co < d.cout; ++co) {
                    const int i = w_off(l) + (tap * d.cin + ci) * d.cout + co;
                    if (ci < d.real_cin && co < d.real_cout) {
                        const double g = std::sqrt(-2.0 * std::log(next())) * std::cos(6.283185307179586 * next());
                        hp[i] = (float)(sd * g);
                        hm[i] = 1.0f;
                    }
                }
        for (int co = 0; co < d.real_cout; ++co) hm[b_off(l) + co] = 1.0f;
    }
    // Every upload and clear goes on the closure's own (non-blocking) stream,
    // so the kernels queued after it see the data: a plain cudaMemcpy from
    // pageable memory may return before its DMA lands, and the legacy stream
    // does not order work on a non-blocking one.
    cudaMemcpyAsync(c->p, hp.data(), P, cudaMemcpyHostToDevice, c->stream);
    cudaMemcpyAsync(c->mask, hm.data(), P, cudaMemcpyHostToDevice, c->stream);
    cudaMemsetAsync(c->m, 0, P, c->stream);
    cudaMemsetAsync(c->v, 0, P, c->stream);
    cudaMemsetAsync(c->g, 0, P, c->stream);
    cudaMemsetAsync(c->err, 0, sizeof(int), c->stream);
    // B images are fully rewritten by pack; zero them once so padding is 0
    for (int l = 0; l < 4; ++l) {
        cudaMemsetAsync(c->fimg[l], 0, cl::bimg_bytes(kLayers[l].cin, kLayers[l].cout), c->stream);
        if (l > 0) cudaMemsetAsync(c->bimg[l], 0, cl::bimg_bytes(kLayers[l].cout, kLayers[l].cin), c->stream);
    }
    int s = pack(c, c->stream);
    if (s == LBMAN_OK) s = upload_scales(c);
    if (s != LBMAN_OK) {
        lbman_closure_destroy(c);
        return s;
    }
    *out = c;
    return LBMAN_OK;
}

int lbman_closure_destroy(lbman_closure* c) {
    if (!c) return LBMAN_OK;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (float* x : c->snaps) cudaFree(x);
    for (float* x : c->targets) cudaFree(x);
    for (float* x : c->rollout_in) cudaFree(x);
    void* ptrs[] = {c->p, c->g, c->m, c->v, c->mask, c->act0, c->gout, c->act[0], c->act[1], c->act[2],
                    c->pre[0], c->pre[1], c->pre[2], c->gbuf[0], c->gbuf[1], c->out, c->wpart, c->bpart,
                    c->lpart, c->loss_hist, c->scales, c->err};
    for (void* x : ptrs) cudaFree(x);
    for (int l = 0; l < 4; ++l) {
        cudaFree(c->fimg[l]);
        cudaFree(c->bimg[l]);
    }
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return LBMAN_OK;
}

int lbman_closure_get_params(lbman_closure* c, float* p) {
    if (!c || !p) return failc(LBMAN_ERR_ARG, "closure: null argument");
    CL_CUDA(cudaSetDevice(c->device));
    CL_CUDA(cudaMemcpy(p, c->p, kNParams * sizeof(float), cudaMemcpyDeviceToHost));
    return LBMAN_OK;
}

int lbman_closure_set_params(lbman_closure* c, const float* p) {
    if (!c || !p) return failc(LBMAN_ERR_ARG, "closure: null argument");
    CL_CUDA(cudaSetDevice(c->device));
    std::vector<float> hm(kNParams), hp(p, p + kNParams);
    CL_CUDA(cudaMemcpy(hm.data(), c->mask, kNParams * sizeof(float), cudaMemcpyDeviceToHost));
    for (int i = 0; i < kNParams; ++i) hp[i] *= hm[i];
    CL_CUDA(cudaMemcpyAsync(c->p, hp.data(), kNParams * sizeof(float), cudaMemcpyHostToDevice, c->stream));
    CL_TRY(pack(c, c->stream));
    CL_CUDA(cudaStreamSynchronize(c->stream));
    return LBMAN_OK;
}

int lbman_closure_get_scales(lbman_closure* c, float* shift9, float* scale9, float* out_scale8) {
    if (!c) return failc(LBMAN_ERR_ARG, "closure: null argument");
    if (shift9) std::memcpy(shift9, c->h_shift, sizeof(c->h_shift));
    if (scale9) std::memcpy(scale9, c->h_scale, sizeof(c->h_scale));
    if (out_scale8) std::memcpy(out_scale8, c->h_out, sizeof(c->h_out));
    return LBMAN_OK;
}

int lbman_closure_set_scales(lbman_closure* c, const float* shift9, const float* scale9, const float* out_scale8) {
    if (!c || !shift9 || !scale9 || !out_scale8) return failc(LBMAN_ERR_ARG, "closure: null argument");
    for (int j = 0; j < 9; ++j)
        if (!(scale9[j] > 0.0f)) return failc(LBMAN_ERR_ARG, "closure: scales must be positive");
    for (int j = 0; j < 8; ++j)
        if (!(out_scale8[j] > 0.0f)) return failc(LBMAN_ERR_ARG, "closure: scales must be positive");
    std::memcpy(c->h_shift, shift9, sizeof(c->h_shift));
    std::memcpy(c->h_scale, scale9, sizeof(c->h_scale));
    std::memcpy(c->h_out, out_scale8, sizeof(c->h_out));
    CL_CUDA(cudaSetDevice(c->device));
    return upload_scales(c);
}

int lbman_closure_forward(lbman_closure* c, const float* feat9, float* out8) {
    if (!c || !feat9 || !out8) return failc(LBMAN_ERR_ARG, "closure: null argument");
    CL_CUDA(cudaSetDevice(c->device));
    const int64_t V = c->V;
    float* dx = nullptr;
    CL_CUDA(cudaMalloc(&dx, 9 * V * sizeof(float)));
    int s = LBMAN_OK;
    if (cudaMemcpyAsync(dx, feat9, 9 * V * sizeof(float), cudaMemcpyHostToDevice, c->stream) != cudaSuccess)
        s = LBMAN_ERR_CUDA;
    if (s == LBMAN_OK) s = features(c, c->stream, dx, dx + V, dx + 4 * V);
    if (s == LBMAN_OK) s = forward(c, c->stream);
    if (s == LBMAN_OK && cudaStreamSynchronize(c->stream) != cudaSuccess) s = LBMAN_ERR_CUDA;
    if (s == LBMAN_OK) s = check_err(c);
    if (s == LBMAN_OK) {
        std::vector<float> o((size_t)V * 16);
        cudaMemcpy(o.data(), c->out, o.size() * 4, cudaMemcpyDeviceToHost);
        for (int64_t i = 0; i < V; ++i)
            for (int j = 0; j < 8; ++j) out8[j * V + i] = o[i * 16 + j];
    }
    cudaFree(dx);
    return s == LBMAN_ERR_CUDA ? failc(s, "closure forward failed") : s;
}

int lbman_closure_gradient(lbman_closure* c, const float* feat9, const float* target8, double* loss, float* grad) {
    if (!c || !feat9 || !target8) return failc(LBMAN_ERR_ARG, "closure: null argument");
    CL_CUDA(cudaSetDevice(c->device));
    const int64_t V = c->V;
    float *dx = nullptr, *dt = nullptr;
    double* dl = nullptr;
    CL_CUDA(cudaMalloc(&dx, 9 * V * sizeof(float)));
    int s = LBMAN_OK;
    if (cudaMalloc(&dt, 8 * V * sizeof(float)) != cudaSuccess || cudaMalloc(&dl, sizeof(double)) != cudaSuccess)
        s = LBMAN_ERR_NOMEM;
    if (s == LBMAN_OK && (cudaMemcpyAsync(dx, feat9, 9 * V * 4, cudaMemcpyHostToDevice, c->stream) != cudaSuccess ||
                          cudaMemcpyAsync(dt, target8, 8 * V * 4, cudaMemcpyHostToDevice, c->stream) != cudaSuccess))
        s = LBMAN_ERR_CUDA;
    if (s == LBMAN_OK) s = features(c, c->stream, dx, dx + V, dx + 4 * V);
    if (s == LBMAN_OK) s = forward(c, c->stream);
    if (s == LBMAN_OK) s = loss_grad(c, c->stream, dt);
    if (s == LBMAN_OK) {
        fold_loss_kernel<<<1, 32, 0, c->stream>>>(c->lpart, c->Gb, 1.0 / (8.0 * (double)V), dl);
        s = backward(c, c->stream);
    }
    if (s == LBMAN_OK && cudaStreamSynchronize(c->stream) != cudaSuccess) s = LBMAN_ERR_CUDA;
    if (s == LBMAN_OK) s = check_err(c);
    if (s == LBMAN_OK) {
        if (loss) cudaMemcpy(loss, dl, sizeof(double), cudaMemcpyDeviceToHost);
        if (grad) cudaMemcpy(grad, c->g, kNParams * sizeof(float), cudaMemcpyDeviceToHost);
    }
    cudaFree(dx);
    cudaFree(dt);
    cudaFree(dl);
    return s == LBMAN_ERR_CUDA ? failc(s, "closure gradient failed") : s;
}

// Box-filters the fine state of v onto the coarse grid as a new snapshot of
// trajectory `traj`.
static int record_view(lbman_closure* c, const SolverView& v, int traj) {
    if (v.prec == LBMAN_FP64) return failc(LBMAN_ERR_UNSUPPORTED, "closure: the fine solver must be FP32 or FP16");
    if (!v.uploaded) return failc(LBMAN_ERR_STATE, "closure: fine solver has no state");
    if (v.nx % c->nx || v.ny % c->ny || v.nz % c->nz || v.nx / c->nx != v.ny / c->ny || v.nx / c->nx != v.nz / c->nz)
        return failc(LBMAN_ERR_ARG, "closure: fine grid is not an integer multiple of the coarse grid");
    const int f = v.nx / c->nx;
    CL_CUDA(cudaSetDevice(c->device));
    float* snap = nullptr;
    CL_CUDA(cudaMalloc(&snap, 9 * c->V * sizeof(float)));
    cl::filter_kernel<<<c->Gb, 256, 0, v.stream>>>(static_cast<const float*>(v.rho), static_cast<const float*>(v.u),
                                                   static_cast<const float*>(v.q), v.nx, v.ny, v.nz, f, snap);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(v.stream);
    if (e != cudaSuccess) {
        cudaFree(snap);
        return cuda_fail(e, "closure record");
    }
    c->cur_traj = std::max(c->cur_traj, traj);
    c->snaps.push_back(snap);
    c->traj.push_back(traj);
    return LBMAN_OK;
}

int lbman_closure_record(lbman_closure* c, lbman_solver* fine, int new_trajectory) {
    if (!c || !fine) return failc(LBMAN_ERR_ARG, "closure: null argument");
    SolverView v;
    CL_TRY(solver_view(fine, &v));
    return record_view(c, v, (new_trajectory || c->cur_traj < 0) ? c->cur_traj + 1 : c->cur_traj);
}

int lbman_closure_record_box(lbman_closure* c, lbman_ensemble* e, int box, int trajectory) {
    if (!c || !e || trajectory < 0) return failc(LBMAN_ERR_ARG, "closure: bad arguments");
    SolverView v;
    CL_TRY(ensemble_box_view(e, box, &v));
    return record_view(c, v, trajectory);
}

int lbman_closure_dataset(lbman_closure* c, int* snapshots, int* pairs) {
    if (!c) return failc(LBMAN_ERR_ARG, "closure: null argument");
    if (snapshots) *snapshots = (int)c->snaps.size();
    if (pairs) *pairs = (int)c->targets.size();
    return LBMAN_OK;
}

int lbman_closure_load_snapshot(lbman_closure* c, int k, lbman_solver* coarse) {
    if (!c || !coarse || k < 0 || k >= (int)c->snaps.size()) return failc(LBMAN_ERR_ARG, "closure: bad snapshot");
    SolverView v;
    if (!coarse_f32(c, coarse, &v)) return failc(LBMAN_ERR_ARG, "closure: coarse solver must be FP32/FP16 on the closure grid");
    const float* x = c->snaps[k];
    CL_TRY(solver_set_state(coarse, x, x + c->V, x + 4 * c->V));
    CL_CUDA(cudaStreamSynchronize(v.stream));
    return LBMAN_OK;
}

// Index of the snapshot recorded `ahead` recordings of the same trajectory
// after snapshot k, or -1.
static int next_of(const lbman_closure* c, int k, int ahead) {
    int n = k;
    for (int left = ahead; left > 0; --left) {
        int j = n + 1;
        while (j < (int)c->snaps.size() && c->traj[j] != c->traj[k]) ++j;
        if (j >= (int)c->snaps.size()) return -1;
        n = j;
    }
    return n;
}

// One corrected coarse step (the operator of lbman_closure_step).
static int corrected_step(lbman_closure* c, lbman_solver* coarse) {
    SolverView w;
    CL_TRY(solver_view(coarse, &w));
    CL_TRY(features(c, w.stream, static_cast<const float*>(w.rho), static_cast<const float*>(w.u),
                    static_cast<const float*>(w.q)));
    CL_TRY(forward(c, w.stream));
    CL_TRY(solver_reset_populations(coarse));
    CL_TRY(lbman_step(coarse, 1));
    CL_TRY(solver_view(coarse, &w));
    cl::apply_kernel<<<c->Gb, 256, 0, w.stream>>>(c->out, c->scales + 18, c->V, c->gain, static_cast<float*>(w.u),
                                                  static_cast<float*>(w.q));
    CL_CUDA(cudaGetLastError());
    return LBMAN_OK;
}

int lbman_closure_add_rollout_pairs(lbman_closure* c, lbman_solver* coarse, int m, int stride, int* added) {
    if (!c || !coarse || m < 1 || stride < 1) return failc(LBMAN_ERR_ARG, "closure: bad arguments");
    SolverView v;
    if (!coarse_f32(c, coarse, &v)) return failc(LBMAN_ERR_ARG, "closure: coarse solver must be FP32/FP16 on the closure grid");
    CL_CUDA(cudaSetDevice(c->device));
    const int64_t V = c->V;
    int count = 0, eligible = 0;
    for (size_t k = 0; k < c->snaps.size(); ++k) {
        const int nk = next_of(c, (int)k, m + 1);
        if (nk < 0 || (eligible++ % stride) != 0) continue;
        // m corrected steps from the filtered fine state: where the corrected
        // run actually is after m steps ...
        const float* x = c->snaps[k];
        CL_TRY(solver_set_state(coarse, x, x + V, x + 4 * V));
        for (int i = 0; i < m; ++i) CL_TRY(corrected_step(c, coarse));
        SolverView w;
        CL_TRY(solver_view(coarse, &w));
        float* in = nullptr;
        CL_CUDA(cudaMalloc(&in, 9 * V * sizeof(float)));
        c->rollout_in.push_back(in);
        CL_CUDA(cudaMemcpyAsync(in, w.rho, V * sizeof(float), cudaMemcpyDeviceToDevice, w.stream));
        CL_CUDA(cudaMemcpyAsync(in + V, w.u, 3 * V * sizeof(float), cudaMemcpyDeviceToDevice, w.stream));
        CL_CUDA(cudaMemcpyAsync(in + 4 * V, w.q, 5 * V * sizeof(float), cudaMemcpyDeviceToDevice, w.stream));
        // ... and the correction that takes its plain step to the filtered
        // fine state one coarse step later
        CL_TRY(solver_set_state(coarse, in, in + V, in + 4 * V));
        CL_TRY(lbman_step(coarse, 1));
        CL_TRY(solver_view(coarse, &w));
        float* t = nullptr;
        CL_CUDA(cudaMalloc(&t, 8 * V * sizeof(float)));
        cl::target_kernel<<<c->Gb, 256, 0, w.stream>>>(c->snaps[nk], static_cast<const float*>(w.u),
                                                        static_cast<const float*>(w.q), V, t);
        CL_CUDA(cudaGetLastError());
        c->targets.push_back(t);
        c->pair_in.push_back(in);
        ++count;
    }
    CL_CUDA(cudaStreamSynchronize(v.stream));
    if (added) *added = count;
    return check_err(c);
}

int lbman_closure_build_targets(lbman_closure* c, lbman_solver* coarse, int fit_scales) {
    if (!c || !coarse) return failc(LBMAN_ERR_ARG, "closure: null argument");
    SolverView v;
    if (!coarse_f32(c, coarse, &v)) return failc(LBMAN_ERR_ARG, "closure: coarse solver must be FP32/FP16 on the closure grid");
    CL_CUDA(cudaSetDevice(c->device));
    for (float* x : c->targets) cudaFree(x);
    for (float* x : c->rollout_in) cudaFree(x);
    c->targets.clear();
    c->pair_in.clear();
    c->rollout_in.clear();
    const int64_t V = c->V;
    for (size_t k = 0; k < c->snaps.size(); ++k) {
        const int nk = next_of(c, (int)k, 1);
        if (nk < 0) continue;
        const float* x = c->snaps[k];
        CL_TRY(solver_set_state(coarse, x, x + V, x + 4 * V));
        CL_TRY(lbman_step(coarse, 1));
        SolverView w;
        CL_TRY(solver_view(coarse, &w));
        float* t = nullptr;
        CL_CUDA(cudaMalloc(&t, 8 * V * sizeof(float)));
        cl::target_kernel<<<c->Gb, 256, 0, w.stream>>>(c->snaps[nk], static_cast<const float*>(w.u),
                                                        static_cast<const float*>(w.q), V, t);
        CL_CUDA(cudaGetLastError());
        c->targets.push_back(t);
        c->pair_in.push_back(x);
    }
    CL_CUDA(cudaStreamSynchronize(v.stream));
    if (fit_scales && !c->targets.empty()) {
        // per-channel mean / std of the inputs, rms of the targets
        double* dp = nullptr;
        CL_CUDA(cudaMalloc(&dp, (size_t)c->Gb * 9 * 2 * sizeof(double)));
        std::vector<double> hp((size_t)c->Gb * 9 * 2), in1(9, 0.0), in2(9, 0.0), t2(8, 0.0);
        double nin = 0.0, nt = 0.0;
        for (size_t k = 0; k < c->snaps.size(); ++k) {
            cl::moments_kernel<<<c->Gb, cl::kThreads, 0, c->stream>>>(c->snaps[k], nullptr, 9, V, dp);
            cudaMemcpyAsync(hp.data(), dp, hp.size() * 8, cudaMemcpyDeviceToHost, c->stream);
            cudaStreamSynchronize(c->stream);
            for (int b = 0; b < c->Gb; ++b)
                for (int j = 0; j < 9; ++j) {
                    in1[j] += hp[((size_t)b * 9 + j) * 2];
                    in2[j] += hp[((size_t)b * 9 + j) * 2 + 1];
                }
            nin += (double)V;
        }
        for (size_t k = 0; k < c->targets.size(); ++k) {
            cl::moments_kernel<<<c->Gb, cl::kThreads, 0, c->stream>>>(c->targets[k], nullptr, 8, V, dp);
            cudaMemcpyAsync(hp.data(), dp, (size_t)c->Gb * 8 * 2 * 8, cudaMemcpyDeviceToHost, c->stream);
            cudaStreamSynchronize(c->stream);
            for (int b = 0; b < c->Gb; ++b)
                for (int j = 0; j < 8; ++j) t2[j] += hp[((size_t)b * 8 + j) * 2 + 1];
            nt += (double)V;
        }
        cudaFree(dp);
        for (int j = 0; j < 9; ++j) {
            const double mu = in1[j] / nin;
            const double var = std::max(in2[j] / nin - mu * mu, 0.0);
            c->h_shift[j] = (float)mu;
            c->h_scale[j] = (float)std::max(std::sqrt(var), 1e-12);
        }
        // Q and u corrections share one scale per field so the output keeps
        // the tensor / vector structure
        double qs = 0.0, us = 0.0;
        for (int j = 0; j < 5; ++j) qs += t2[j];
        for (int j = 5; j < 8; ++j) us += t2[j];
        const float qsc = (float)std::max(std::sqrt(qs / (5.0 * nt)), 1e-12);
        const float usc = (float)std::max(std::sqrt(us / (3.0 * nt)), 1e-12);
        for (int j = 0; j < 5; ++j) c->h_out[j] = qsc;
        for (int j = 5; j < 8; ++j) c->h_out[j] = usc;
        CL_TRY(upload_scales(c));
    }
    return LBMAN_OK;
}

int lbman_closure_train(lbman_closure* c, int iters, float lr, uint64_t seed, double* loss_first,
                        double* loss_last) {
    if (!c || iters < 1 || !(lr > 0.0f)) return failc(LBMAN_ERR_ARG, "closure: bad arguments");
    if (c->targets.empty()) return failc(LBMAN_ERR_STATE, "closure: no training pairs (record and build targets)");
    CL_CUDA(cudaSetDevice(c->device));
    if (c->loss_cap < iters) {
        cudaFree(c->loss_hist);
        c->loss_hist = nullptr;
        CL_CUDA(cudaMalloc(&c->loss_hist, (size_t)iters * sizeof(double)));
        c->loss_cap = iters;
    }
    const int64_t V = c->V;
    const int npairs = (int)c->targets.size();
    uint64_t st = seed * 0x9e3779b97f4a7c15ull + 1;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int it = 0; it < iters; ++it) {
        st ^= st << 13;
        st ^= st >> 7;
        st ^= st << 17;
        const int pi = (int)(st % (uint64_t)npairs);
        const float* x = c->pair_in[pi];
        CL_TRY(features(c, c->stream, x, x + V, x + 4 * V, c->train_noise, st));
        CL_TRY(forward(c, c->stream));
        CL_TRY(loss_grad(c, c->stream, c->targets[pi]));
        fold_loss_kernel<<<1, 32, 0, c->stream>>>(c->lpart, c->Gb, 1.0 / (8.0 * (double)V), c->loss_hist + it);
        CL_TRY(backward(c, c->stream));
        ++c->adam_t;
        const float bc1 = 1.0f - std::pow(b1, (float)c->adam_t), bc2 = 1.0f - std::pow(b2, (float)c->adam_t);
        cl::adam_kernel<<<64, 256, 0, c->stream>>>(c->p, c->g, c->m, c->v, c->mask, kNParams, lr, b1, b2, eps, bc1,
                                                   bc2);
        CL_CUDA(cudaGetLastError());
        CL_TRY(pack(c, c->stream));
    }
    CL_CUDA(cudaStreamSynchronize(c->stream));
    CL_TRY(check_err(c));
    std::vector<double> h((size_t)iters);
    CL_CUDA(cudaMemcpy(h.data(), c->loss_hist, h.size() * sizeof(double), cudaMemcpyDeviceToHost));
    const int w = std::max(1, iters / 10);
    double a = 0.0, b = 0.0;
    for (int i = 0; i < w; ++i) {
        a += h[i];
        b += h[iters - 1 - i];
    }
    if (loss_first) *loss_first = a / w;
    if (loss_last) *loss_last = b / w;
    return LBMAN_OK;
}

static_assert(LBMAN_CLOSURE_WAIT_DEFAULT == lbman::tc::kWaitLimit, "the header's default is the kernels' limit");

int lbman_closure_set_wait_limit(lbman_closure* c, uint32_t polls) {
    if (!c) return failc(LBMAN_ERR_ARG, "closure: null handle");
    c->wait_limit = polls;
    return LBMAN_OK;
}

int lbman_closure_set_options(lbman_closure* c, float train_noise, float gain) {
    if (!c || !(train_noise >= 0.0f) || !(gain >= 0.0f)) return failc(LBMAN_ERR_ARG, "closure: bad options");
    c->train_noise = train_noise;
    c->gain = gain;
    return LBMAN_OK;
}

int lbman_closure_step(lbman_closure* c, lbman_solver* coarse, int nsteps) {
    if (!c || !coarse || nsteps < 0) return failc(LBMAN_ERR_ARG, "closure: bad arguments");
    SolverView v;
    if (!coarse_f32(c, coarse, &v)) return failc(LBMAN_ERR_ARG, "closure: coarse solver must be FP32/FP16 on the closure grid");
    if (!v.uploaded) return failc(LBMAN_ERR_STATE, "closure: coarse solver has no state");
    CL_CUDA(cudaSetDevice(c->device));
    for (int n = 0; n < nsteps; ++n) CL_TRY(corrected_step(c, coarse));
    CL_CUDA(cudaStreamSynchronize(v.stream));
    return check_err(c);
}

}  // extern "C"

extern "C" int lbman_closure_selftest(int device, double* max_rel_err) {
    using namespace lbman;
    if (cudaSetDevice(device) != cudaSuccess) return LBMAN_ERR_CUDA;
    const int M = kSelfM, N = kSelfN, K = kSelfK;
    std::vector<float> A(M * K), B(N * K), D(M * N);
    uint64_t s = 0x9e3779b97f4a7c15ull;
    auto rnd = [&]() {
        s ^= s << 13; s ^= s >> 7; s ^= s << 17;
        return (float)((double)(s >> 11) * 0x1.0p-53 * 2.0 - 1.0);
    };
    for (auto& x : A) x = bf16_round(rnd());
    for (auto& x : B) x = bf16_round(rnd());
    float *dA = nullptr, *dB = nullptr, *dD = nullptr;
    int* derr = nullptr;
    int status = LBMAN_OK;
    if (cudaMalloc(&dA, A.size() * 4) != cudaSuccess || cudaMalloc(&dB, B.size() * 4) != cudaSuccess ||
        cudaMalloc(&dD, D.size() * 4) != cudaSuccess || cudaMalloc(&derr, sizeof(int)) != cudaSuccess)
        status = LBMAN_ERR_NOMEM;
    if (status == LBMAN_OK) {
        cudaMemcpy(dA, A.data(), A.size() * 4, cudaMemcpyHostToDevice);
        cudaMemcpy(dB, B.data(), B.size() * 4, cudaMemcpyHostToDevice);
        cudaFuncSetAttribute(tc_selftest_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSelfSmem);
    }
    for (int combo = 0; combo < 4 && status == LBMAN_OK; ++combo) {
        const int a_mn = combo & 1, b_mn = combo >> 1;
        cudaMemset(dD, 0xFF, D.size() * 4);
        cudaMemset(derr, 0, sizeof(int));
        tc_selftest_kernel<<<1, 128, kSelfSmem>>>(dA, dB, dD, a_mn, b_mn, derr);
        if (cudaDeviceSynchronize() != cudaSuccess) {
            status = LBMAN_ERR_CUDA;
            break;
        }
        int herr = 0;
        cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost);
        cudaMemcpy(D.data(), dD, D.size() * 4, cudaMemcpyDeviceToHost);
        double worst = 0.0;
        for (int m = 0; m < M; ++m)
            for (int n = 0; n < N; ++n) {
                double ref = 0.0, mag = 0.0;
                for (int k = 0; k < K; ++k) {
                    ref += (double)A[m * K + k] * B[n * K + k];
                    mag += std::fabs((double)A[m * K + k] * B[n * K + k]);
                }
                const double e = std::fabs(D[m * N + n] - ref) / (mag > 0 ? mag : 1.0);
                if (!(e <= worst)) worst = e;  // NaN propagates
            }
        if (max_rel_err) max_rel_err[combo] = herr ? -1.0 : worst;
        if (herr) status = LBMAN_ERR_TIMEOUT;
    }
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dD);
    cudaFree(derr);
    return status;
}
