// stats.cu -- flow and order statistics of one box: kinetic-energy spectrum,
// Q-tensor autocorrelation and correlation length, mean / rms speed.  No
// counterpart in the reference (its analysis stops at the defect finder,
// src/analysis/defect_finder.tpp); definitions are stated in stats.h and in
// the C header.
//
// Transforms are cuFFT 3D real-to-complex (library FFTs, like cuBLAS for a
// plain GEMM); the power accumulation and the shell binning are kernels of
// this file.  Shell sums are accumulated in FP64: per block in shared memory,
// then folded over blocks in a fixed order.
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "stats.h"

namespace lbman {
namespace stats {

namespace {

constexpr int kThreads = 256;

// P = |A|^2 (mode 0), P += |A|^2 (1), P = 2|A|^2 + 2|B|^2 + 2 Re(A conj B) (2),
// P += 2|A|^2 (3).
template <class R, class C>
__global__ void __launch_bounds__(kThreads) power_kernel(const C* __restrict__ A, const C* __restrict__ B,
                                                         R* __restrict__ P, int64_t n, int mode) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const C a = A[i];
        const R pa = a.x * a.x + a.y * a.y;
        if (mode == 0) {
            P[i] = pa;
        } else if (mode == 1) {
            P[i] += pa;
        } else if (mode == 2) {
            const C b = B[i];
            P[i] = R(2) * pa + R(2) * (b.x * b.x + b.y * b.y) + R(2) * (a.x * b.x + a.y * b.y);
        } else {
            P[i] += R(2) * pa;
        }
    }
}

// (value, count) per shell for this block into partials[(q*nbins + b)*G + block].
__device__ void flush_bins(const double* sv, const double* sc, int nbins, double* partials, int G) {
    for (int b = threadIdx.x; b < nbins; b += blockDim.x) {
        partials[(size_t)b * G + blockIdx.x] = sv[b];
        partials[((size_t)nbins + b) * G + blockIdx.x] = sc[b];
    }
}

// Half-spectrum modes (kz, ky, kx <= nx/2) into wavenumber shells
// b = round(nmax * |(m_x/nx, m_y/ny, m_z/nz)|); modes with 0 < kx < nx/2
// stand for their conjugate partner too (weight 2).
template <class R>
__global__ void __launch_bounds__(kThreads) kshell_kernel(const R* __restrict__ P, int nx, int ny, int nz, int nbins,
                                                          double* __restrict__ partials) {
    extern __shared__ double sh[];
    double* sv = sh;
    double* sc = sh + nbins;
    for (int b = threadIdx.x; b < 2 * nbins; b += blockDim.x) sh[b] = 0.0;
    __syncthreads();
    const int nh = nx / 2 + 1;
    const int64_t n = (int64_t)nz * ny * nh;
    const double nmax = (double)max(nx, max(ny, nz));
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int kx = (int)(i % nh);
        const int64_t t = i / nh;
        const int ky = (int)(t % ny), kz = (int)(t / ny);
        const int my = ky <= ny / 2 ? ky : ky - ny;
        const int mz = kz <= nz / 2 ? kz : kz - nz;
        const double fx = (double)kx / nx, fy = (double)my / ny, fz = (double)mz / nz;
        const int b = (int)(nmax * sqrt(fx * fx + fy * fy + fz * fz) + 0.5);
        if (b < nbins) {
            const double w = (kx == 0 || 2 * kx == nx) ? 1.0 : 2.0;
            atomicAdd(&sv[b], w * (double)P[i]);
            atomicAdd(&sc[b], w);
        }
    }
    __syncthreads();
    flush_bins(sv, sc, nbins, partials, gridDim.x);
}

// Real-space separations r (minimum image on every axis) into shells
// b = round(|r|).
template <class R>
__global__ void __launch_bounds__(kThreads) rshell_kernel(const R* __restrict__ Gr, int nx, int ny, int nz, int nbins,
                                                          double* __restrict__ partials) {
    extern __shared__ double sh[];
    double* sv = sh;
    double* sc = sh + nbins;
    for (int b = threadIdx.x; b < 2 * nbins; b += blockDim.x) sh[b] = 0.0;
    __syncthreads();
    const int64_t n = (int64_t)nz * ny * nx;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(i % nx);
        const int64_t t = i / nx;
        const int y = (int)(t % ny), z = (int)(t / ny);
        const double dx = min(x, nx - x), dy = min(y, ny - y), dz = min(z, nz - z);
        const int b = (int)(sqrt(dx * dx + dy * dy + dz * dz) + 0.5);
        if (b < nbins) {
            atomicAdd(&sv[b], (double)Gr[i]);
            atomicAdd(&sc[b], 1.0);
        }
    }
    __syncthreads();
    flush_bins(sv, sc, nbins, partials, gridDim.x);
}

// Real array -> complex array with zero imaginary parts.
template <class R, class C>
__global__ void __launch_bounds__(kThreads) to_complex_kernel(const R* __restrict__ P, C* __restrict__ A, int64_t n) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        C c;
        c.x = P[i];
        c.y = R(0);
        A[i] = c;
    }
}

// out[j] = sum over blocks g (in order) of partials[j*G + g].
__global__ void __launch_bounds__(kThreads) fold_bins_kernel(const double* __restrict__ partials, int G, int n,
                                                             double* __restrict__ out) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    double acc = 0.0;
    for (int g = 0; g < G; ++g) acc += partials[(size_t)j * G + g];
    out[j] = acc;
}

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Per block: sum |u| and sum |u|^2 into partials[q*G + block].
template <class R>
__global__ void __launch_bounds__(kThreads) speed_kernel(const R* __restrict__ u, int64_t V,
                                                         double* __restrict__ partials) {
    __shared__ double sh[2][kThreads / 32];
    double s1 = 0.0, s2 = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < V; i += (int64_t)gridDim.x * blockDim.x) {
        const double ux = u[i], uy = u[V + i], uz = u[2 * V + i];
        const double u2 = ux * ux + uy * uy + uz * uz;
        s1 += sqrt(u2);
        s2 += u2;
    }
    s1 = warp_sum_d(s1);
    s2 = warp_sum_d(s2);
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        sh[0][w] = s1;
        sh[1][w] = s2;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int k = 0; k < kThreads / 32; ++k) {
            a += sh[0][k];
            b += sh[1][k];
        }
        partials[blockIdx.x] = a;
        partials[gridDim.x + blockIdx.x] = b;
    }
}

}  // namespace

struct Workspace {
    int nx = 0, ny = 0, nz = 0, G = 0;
    bool dbl = false;
    int64_t V = 0, NC = 0;
    cufftHandle r2c = 0, c2r = 0;
    bool plans = false;
    void* A = nullptr;     // complex NC
    void* B = nullptr;     // complex NC (also the real C2R output)
    void* Rin = nullptr;   // real V: copy of the transformed component
    void* P = nullptr;     // real NC: accumulated power
    double* partials = nullptr;
    size_t partials_cap = 0;
    double* out = nullptr;  // device, 2 * kMaxBins
};

#define ST_CUDA(x)                                  \
    do {                                            \
        cudaError_t e_ = (x);                       \
        if (e_ != cudaSuccess) return (int)e_;      \
    } while (0)
#define ST_FFT(x)                                   \
    do {                                            \
        cufftResult r_ = (x);                       \
        if (r_ != CUFFT_SUCCESS) return 1000 + (int)r_; \
    } while (0)

Workspace* create(int nx, int ny, int nz, bool dbl, int num_sms) {
    Workspace* w = new Workspace;
    w->nx = nx;
    w->ny = ny;
    w->nz = nz;
    w->dbl = dbl;
    w->V = (int64_t)nx * ny * nz;
    w->NC = (int64_t)nz * ny * (nx / 2 + 1);
    w->G = 2 * std::max(1, num_sms);
    return w;
}

void destroy(Workspace* w) {
    if (!w) return;
    if (w->plans) {
        cufftDestroy(w->r2c);
        cufftDestroy(w->c2r);
    }
    cudaFree(w->A);
    cudaFree(w->B);
    cudaFree(w->Rin);
    cudaFree(w->P);
    cudaFree(w->partials);
    cudaFree(w->out);
    delete w;
}

namespace {

int ensure(Workspace* w, int nbins, cudaStream_t st) {
    const size_t rb = w->dbl ? 8 : 4;
    if (!w->plans) {
        ST_FFT(cufftPlan3d(&w->r2c, w->nz, w->ny, w->nx, w->dbl ? CUFFT_D2Z : CUFFT_R2C));
        ST_FFT(cufftPlan3d(&w->c2r, w->nz, w->ny, w->nx, w->dbl ? CUFFT_Z2D : CUFFT_C2R));
        w->plans = true;
        ST_CUDA(cudaMalloc(&w->A, (size_t)w->NC * 2 * rb));
        ST_CUDA(cudaMalloc(&w->B, (size_t)w->NC * 2 * rb));
        ST_CUDA(cudaMalloc(&w->Rin, (size_t)w->V * rb));
        ST_CUDA(cudaMalloc(&w->P, (size_t)w->NC * rb));
        ST_CUDA(cudaMalloc(&w->out, 2 * (size_t)kMaxBins * sizeof(double)));
        ST_CUDA(cudaFuncSetAttribute(kshell_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     2 * kMaxBins * (int)sizeof(double)));
        ST_CUDA(cudaFuncSetAttribute(kshell_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     2 * kMaxBins * (int)sizeof(double)));
        ST_CUDA(cudaFuncSetAttribute(rshell_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     2 * kMaxBins * (int)sizeof(double)));
        ST_CUDA(cudaFuncSetAttribute(rshell_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     2 * kMaxBins * (int)sizeof(double)));
    }
    ST_FFT(cufftSetStream(w->r2c, st));
    ST_FFT(cufftSetStream(w->c2r, st));
    const size_t need = (size_t)w->G * 2 * std::max(nbins, 2);
    if (need > w->partials_cap) {
        cudaFree(w->partials);
        w->partials = nullptr;
        ST_CUDA(cudaMalloc(&w->partials, need * sizeof(double)));
        w->partials_cap = need;
    }
    return 0;
}

// Forward transform of one component (copied first: cuFFT may use its
// input as scratch) into dst.
int forward(Workspace* w, const void* comp, void* dst, cudaStream_t st) {
    const size_t rb = w->dbl ? 8 : 4;
    ST_CUDA(cudaMemcpyAsync(w->Rin, comp, (size_t)w->V * rb, cudaMemcpyDeviceToDevice, st));
    if (w->dbl)
        ST_FFT(cufftExecD2Z(w->r2c, (cufftDoubleReal*)w->Rin, (cufftDoubleComplex*)dst));
    else
        ST_FFT(cufftExecR2C(w->r2c, (cufftReal*)w->Rin, (cufftComplex*)dst));
    return 0;
}

int power(Workspace* w, const void* A, const void* B, int mode, cudaStream_t st) {
    const int grid = w->G * 4;
    if (w->dbl)
        power_kernel<double, cufftDoubleComplex><<<grid, kThreads, 0, st>>>(
            (const cufftDoubleComplex*)A, (const cufftDoubleComplex*)B, (double*)w->P, w->NC, mode);
    else
        power_kernel<float, cufftComplex><<<grid, kThreads, 0, st>>>((const cufftComplex*)A, (const cufftComplex*)B,
                                                                     (float*)w->P, w->NC, mode);
    ST_CUDA(cudaGetLastError());
    return 0;
}

int fold_to_host(Workspace* w, int nbins, double* v_host, double* c_host, cudaStream_t st) {
    const int n = 2 * nbins;
    fold_bins_kernel<<<(n + kThreads - 1) / kThreads, kThreads, 0, st>>>(w->partials, w->G, n, w->out);
    ST_CUDA(cudaGetLastError());
    std::vector<double> tmp((size_t)n);
    ST_CUDA(cudaMemcpyAsync(tmp.data(), w->out, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st));
    ST_CUDA(cudaStreamSynchronize(st));
    std::memcpy(v_host, tmp.data(), (size_t)nbins * sizeof(double));
    if (c_host) std::memcpy(c_host, tmp.data() + nbins, (size_t)nbins * sizeof(double));
    return 0;
}

}  // namespace

int velocity_spectrum(Workspace* w, const void* u3, int nbins, double* E, double* counts, cudaStream_t st) {
    if (int r = ensure(w, nbins, st)) return r;
    const size_t rb = w->dbl ? 8 : 4;
    for (int c = 0; c < 3; ++c) {
        if (int r = forward(w, (const char*)u3 + (size_t)c * w->V * rb, w->A, st)) return r;
        if (int r = power(w, w->A, nullptr, c == 0 ? 0 : 1, st)) return r;
    }
    const size_t smem = 2 * (size_t)nbins * sizeof(double);
    if (w->dbl)
        kshell_kernel<double><<<w->G, kThreads, smem, st>>>((const double*)w->P, w->nx, w->ny, w->nz, nbins,
                                                            w->partials);
    else
        kshell_kernel<float><<<w->G, kThreads, smem, st>>>((const float*)w->P, w->nx, w->ny, w->nz, nbins,
                                                           w->partials);
    ST_CUDA(cudaGetLastError());
    if (int r = fold_to_host(w, nbins, E, counts, st)) return r;
    const double norm = 0.5 / ((double)w->V * (double)w->V);
    for (int b = 0; b < nbins; ++b) E[b] *= norm;
    return 0;
}

int q_correlation(Workspace* w, const void* q5, int nbins, double* C, double* counts, cudaStream_t st) {
    if (int r = ensure(w, nbins, st)) return r;
    const size_t rb = w->dbl ? 8 : 4;
    auto comp = [&](int k) { return (const char*)q5 + (size_t)k * w->V * rb; };
    // Q:Q' = 2 xx xx' + 2 yy yy' + xx yy' + yy xx' + 2 (xy xy' + xz xz' + yz yz')
    // (qzz = -qxx - qyy), so its power is 2|X|^2 + 2|Y|^2 + 2 Re(X conj Y) + 2|.|^2 ...
    if (int r = forward(w, comp(0), w->A, st)) return r;
    if (int r = forward(w, comp(3), w->B, st)) return r;
    if (int r = power(w, w->A, w->B, 2, st)) return r;
    for (int k : {1, 2, 4}) {
        if (int r = forward(w, comp(k), w->A, st)) return r;
        if (int r = power(w, w->A, nullptr, 3, st)) return r;
    }
    // P as a complex array (imaginary part 0) -> inverse transform -> the
    // autocorrelation sum V^2 <Q(x):Q(x+r)> at every separation r.
    const int64_t NC = w->NC;
    if (w->dbl) {
        to_complex_kernel<double, cufftDoubleComplex><<<w->G * 4, kThreads, 0, st>>>(
            (const double*)w->P, (cufftDoubleComplex*)w->A, NC);
        ST_CUDA(cudaGetLastError());
        ST_FFT(cufftExecZ2D(w->c2r, (cufftDoubleComplex*)w->A, (cufftDoubleReal*)w->B));
    } else {
        to_complex_kernel<float, cufftComplex><<<w->G * 4, kThreads, 0, st>>>((const float*)w->P,
                                                                              (cufftComplex*)w->A, NC);
        ST_CUDA(cudaGetLastError());
        ST_FFT(cufftExecC2R(w->c2r, (cufftComplex*)w->A, (cufftReal*)w->B));
    }
    const size_t smem = 2 * (size_t)nbins * sizeof(double);
    if (w->dbl)
        rshell_kernel<double><<<w->G, kThreads, smem, st>>>((const double*)w->B, w->nx, w->ny, w->nz, nbins,
                                                            w->partials);
    else
        rshell_kernel<float><<<w->G, kThreads, smem, st>>>((const float*)w->B, w->nx, w->ny, w->nz, nbins,
                                                           w->partials);
    ST_CUDA(cudaGetLastError());
    std::vector<double> cnt((size_t)nbins);
    if (int r = fold_to_host(w, nbins, C, cnt.data(), st)) return r;
    // Shell means normalised by the r = 0 value (shell 0 holds r = 0 alone).
    const double g0 = cnt[0] > 0 ? C[0] / cnt[0] : 0.0;
    for (int b = 0; b < nbins; ++b) C[b] = (cnt[b] > 0 && g0 != 0.0) ? (C[b] / cnt[b]) / g0 : 0.0;
    if (counts) std::memcpy(counts, cnt.data(), (size_t)nbins * sizeof(double));
    return 0;
}

int speed_moments(Workspace* w, const void* u3, double* mean_speed, double* mean_speed2, cudaStream_t st) {
    if (int r = ensure(w, 2, st)) return r;
    if (w->dbl)
        speed_kernel<double><<<w->G, kThreads, 0, st>>>((const double*)u3, w->V, w->partials);
    else
        speed_kernel<float><<<w->G, kThreads, 0, st>>>((const float*)u3, w->V, w->partials);
    ST_CUDA(cudaGetLastError());
    fold_bins_kernel<<<1, kThreads, 0, st>>>(w->partials, w->G, 2, w->out);
    ST_CUDA(cudaGetLastError());
    double r[2];
    ST_CUDA(cudaMemcpyAsync(r, w->out, sizeof(r), cudaMemcpyDeviceToHost, st));
    ST_CUDA(cudaStreamSynchronize(st));
    *mean_speed = r[0] / (double)w->V;
    *mean_speed2 = r[1] / (double)w->V;
    return 0;
}

bool is_nomem(int code) {
    return code == (int)cudaErrorMemoryAllocation || code == 1000 + (int)CUFFT_ALLOC_FAILED;
}

const char* err_string(int code) {
    if (code >= 1000) {
        switch (code - 1000) {
            case CUFFT_ALLOC_FAILED: return "cuFFT: allocation failed";
            case CUFFT_INVALID_VALUE: return "cuFFT: invalid value";
            case CUFFT_INVALID_SIZE: return "cuFFT: invalid size";
            case CUFFT_EXEC_FAILED: return "cuFFT: execution failed";
            case CUFFT_SETUP_FAILED: return "cuFFT: setup failed";
            default: return "cuFFT error";
        }
    }
    return cudaGetErrorString((cudaError_t)code);
}

}  // namespace stats
}  // namespace lbman
