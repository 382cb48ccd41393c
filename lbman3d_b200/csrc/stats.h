// stats.h -- flow and order statistics of one box (no counterpart in the
// reference): the shell-averaged kinetic-energy spectrum, the radially
// averaged Q-tensor autocorrelation with its correlation length, and the
// mean / rms speed.  Fields are the solver's device arrays (x fastest,
// component blocks of V values) in FP64 (dbl) or FP32.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace lbman {
namespace stats {

struct Workspace;  // cuFFT plans and scratch, created on first use

Workspace* create(int nx, int ny, int nz, bool dbl, int num_sms);
void destroy(Workspace* w);

// Each returns a cudaError_t-like code: 0 on success, else a CUDA error or
// cufftResult offset by 1000 (err_string turns it into text).
int velocity_spectrum(Workspace* w, const void* u3, int nbins, double* E_host, double* counts_host,
                      cudaStream_t st);
int q_correlation(Workspace* w, const void* q5, int nbins, double* C_host, double* counts_host,
                  cudaStream_t st);
int speed_moments(Workspace* w, const void* u3, double* mean_speed, double* mean_speed2, cudaStream_t st);
const char* err_string(int code);
bool is_nomem(int code);

// Largest nbins the binning kernels accept.
constexpr int kMaxBins = 8192;

}  // namespace stats
}  // namespace lbman
