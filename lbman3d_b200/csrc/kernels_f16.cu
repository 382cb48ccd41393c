// kernels_f16.cu -- FP32 compute with populations stored as FP16 deviations
// f_i - w_i*rho0; Q, u, rho and the body force are FP32.
#include "kernels_impl.cuh"

LBMAN_DEFINE_LAUNCHERS(f16, float, __half, true)
