// kernels_f32.cu -- FP32 compute with populations stored as FP32 deviations
// f_i - w_i*rho0; Q, u, rho and the body force are FP32.
#include "kernels_impl.cuh"

LBMAN_DEFINE_LAUNCHERS(f32, float, float, true)
