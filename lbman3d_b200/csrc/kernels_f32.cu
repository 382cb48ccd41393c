// kernels_f32.cu -- FP32 compute; populations stored as FP32 (f32) or FP16
// (f16) deviations f_i - w_i*rho0.  Q, u, rho and the body force are FP32.
#include "kernels_impl.cuh"

LBMAN_DEFINE_LAUNCHERS(f32, float, float, true)
LBMAN_DEFINE_LAUNCHERS(f16, float, __half, true)
