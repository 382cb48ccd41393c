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
// process exits.  Host code cannot use the symbol's name as a device address:
// every call fetches the address with cudaGetSymbolAddress while the caller's
// device is current and passes it to the kernels.  The lookup is a table
// search inside the CUDA runtime (no allocation), and doing it per call keeps
// the address right when the device's context was torn down and re-created
// (cudaDeviceReset reloads the module, and the array can move).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstring>

#include "../../include/lbman3d.h"
#include "reduce.cuh"

namespace lbman {
void set_last_error(const char* msg);  // api.cu
}

namespace {

using namespace lbman;

constexpr int kMaxBlocks = LBMAN_NOALLOC_MAX_BLOCKS;

static __device__ __align__(256) double g_partials[kMaxBlocks * kFlowQ];
static __device__ __align__(256) double g_result[16];

int fail(int code, const char* msg) {
    lbman::set_last_error(msg);  // reported by lbman_last_error()
    return code;
}

// Device addresses of the scratch arrays in the current device's context.
int scratch_for_current_device(double** partials, double** result) {
    if (cudaGetSymbolAddress((void**)partials, g_partials) != cudaSuccess ||
        cudaGetSymbolAddress((void**)result, g_result) != cudaSuccess)
        return fail(LBMAN_ERR_CUDA, "cudaGetSymbolAddress of the reduction scratch failed");
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
    // An error left pending by earlier, unrelated work is the caller's to
    // see: report it without clearing it, so the launch checks below see only
    // this call's launches.
    if (cudaPeekAtLastError() != cudaSuccess)
        return fail(LBMAN_ERR_CUDA, "a CUDA error was already pending before the call");
    double* partials = nullptr;
    double* result = nullptr;
    if (int st = scratch_for_current_device(&partials, &result)) return st;

    SimParams P;
    std::memset(&P, 0, sizeof(P));
    P.V = ncells;
    P.c0 = 0;
    P.c1 = ncells;  // the reduction's cell range
    const int G = (int)((ncells + kRedThreads - 1) / kRedThreads < kMaxBlocks
                            ? (ncells + kRedThreads - 1) / kRedThreads
                            : kMaxBlocks);
    cudaStream_t st = (cudaStream_t)cuda_stream;
    if (precision == LBMAN_FP64)
        flow_reduce_kernel<double><<<G, kRedThreads, 0, st>>>(P, (const double*)rho, (const double*)u3,
                                                               (double*)upast3, partials);
    else
        flow_reduce_kernel<float><<<G, kRedThreads, 0, st>>>(P, (const float*)rho, (const float*)u3,
                                                             (float*)upast3, partials);
    if (cudaGetLastError() != cudaSuccess) return fail(LBMAN_ERR_CUDA, "flow reduction launch failed");
    // Every partial the fold reads, and every result slot copied back, is
    // written earlier in this call, so nothing has to be cleared first.
    fold_partials_kernel<<<1, 1024, 0, st>>>(partials, G, kFlowQ, 1, result);
    if (cudaGetLastError() != cudaSuccess) return fail(LBMAN_ERR_CUDA, "fold launch failed");
    double r[kFlowQ];
    if (cudaMemcpyAsync(r, result, sizeof(r), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
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
