// noalloc.cu -- lbman_flow_reduce_noalloc: the flow diagnostics of
// lbman_reduce (mass, momentum, kinetic energy, relative change, max |u|)
// over caller-owned device fields, with every byte of scratch taken from a
// fixed array compiled into the library instead of from cudaMalloc.
//
// Who needs it: code that hosts this library inside a framework whose
// allocator has already reserved (nearly) all device memory, where one more
// cudaMalloc fails or fragments the pool, and time-stepping loops that must
// not call cudaMalloc/cudaFree between steps because cudaFree synchronises
// the whole device.  Those callers own their fields and pass them in; this
// entry point then needs no memory of its own.
//
// The scratch is g_partials below: one FP64 partial sum per reduction block
// and quantity, plus g_result for the folded totals.  It is a __device__
// array, so every GPU that loads the library holds it (about 76 KB) until the
// process exits.  Host code cannot use the symbol's name as a device address;
// the address is fetched once per device with cudaGetSymbolAddress while that
// device is current (on the first call made on it) and passed to the kernels.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "../../include/lbman3d.h"
#include "reduce.cuh"

namespace lbman {
void set_last_error(const char* msg);  // api.cu
}

namespace {

using namespace lbman;

constexpr int kMaxBlocks = LBMAN_NOALLOC_MAX_BLOCKS;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) double g_partials[kMaxBlocks * kFlowQ];
static __device__ __align__(256) double g_result[16];

struct DeviceScratch {
    double* partials = nullptr;
    double* result = nullptr;
    bool ready = false;
};
DeviceScratch g_dev[kMaxDevices];
std::mutex g_mu;

int fail(int code, const char* msg) {
    lbman::set_last_error(msg);  // reported by lbman_last_error()
    return code;
}

// Device addresses of the scratch arrays for the current device.
int scratch_for_current_device(DeviceScratch** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(LBMAN_ERR_CUDA, "cudaGetDevice failed");
    if (dev < 0 || dev >= kMaxDevices) return fail(LBMAN_ERR_UNSUPPORTED, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_mu);
    DeviceScratch& d = g_dev[dev];
    if (!d.ready) {
        cudaError_t e1 = cudaGetSymbolAddress((void**)&d.partials, g_partials);
        cudaError_t e2 = cudaGetSymbolAddress((void**)&d.result, g_result);
        if (e1 != cudaSuccess || e2 != cudaSuccess) {
            d.partials = d.result = nullptr;
            return fail(LBMAN_ERR_CUDA, "cudaGetSymbolAddress of the reduction scratch failed");
        }
        d.ready = true;
    }
    *out = &d;
    return LBMAN_OK;
}

}  // namespace

extern "C" int lbman_flow_reduce_noalloc(int64_t ncells, int precision, const void* rho, const void* u3,
                                         void* upast3, void* cuda_stream, lbman_diag* out) {
    if (!rho || !u3 || !upast3 || !out) return fail(LBMAN_ERR_ARG, "rho, u3, upast3 and out are required");
    if (ncells < 1 || ncells > LBMAN_NOALLOC_MAX_CELLS)
        return fail(LBMAN_ERR_ARG, "ncells must be in [1, LBMAN_NOALLOC_MAX_CELLS]");
    if (precision != LBMAN_FP64 && precision != LBMAN_FP32)
        return fail(LBMAN_ERR_ARG, "precision must be LBMAN_FP64 (double fields) or LBMAN_FP32 (float fields)");
    DeviceScratch* d = nullptr;
    if (int st = scratch_for_current_device(&d)) return st;

    SimParams P;
    std::memset(&P, 0, sizeof(P));
    P.V = ncells;
    const int G = (int)((ncells + kRedThreads - 1) / kRedThreads < kMaxBlocks
                            ? (ncells + kRedThreads - 1) / kRedThreads
                            : kMaxBlocks);
    cudaStream_t st = (cudaStream_t)cuda_stream;
    if (precision == LBMAN_FP64)
        flow_reduce_kernel<double><<<G, kRedThreads, 0, st>>>(P, (const double*)rho, (const double*)u3,
                                                               (double*)upast3, d->partials);
    else
        flow_reduce_kernel<float><<<G, kRedThreads, 0, st>>>(P, (const float*)rho, (const float*)u3,
                                                             (float*)upast3, d->partials);
    // Every partial the fold reads, and every result slot copied back, is
    // written earlier in this call, so nothing has to be cleared first.
    fold_partials_kernel<<<1, 1024, 0, st>>>(d->partials, G, kFlowQ, 1, d->result);
    if (cudaGetLastError() != cudaSuccess) return fail(LBMAN_ERR_CUDA, "reduction launch failed");
    double r[kFlowQ];
    if (cudaMemcpyAsync(r, d->result, sizeof(r), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
        cudaStreamSynchronize(st) != cudaSuccess)
        return fail(LBMAN_ERR_CUDA, "copy of the reduction result failed");
    std::memset(out, 0, sizeof(*out));
    out->mass = r[0]; out->px = r[1]; out->py = r[2]; out->pz = r[3];
    out->kinetic_energy = r[4]; out->rel_change_num = r[5]; out->rel_change_den = r[6]; out->umax2 = r[7];
    out->defect_faces = -1;
    out->nan_detected = std::isnan(r[0]) || std::isnan(r[1]) || std::isnan(r[2]) || std::isnan(r[3]);
    if (out->nan_detected) return fail(LBMAN_ERR_DIVERGED, "NaN in the global mass or momentum");
    return LBMAN_OK;
}
