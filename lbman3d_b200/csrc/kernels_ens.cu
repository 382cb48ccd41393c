// kernels_ens.cu -- ensemble launchers for FP32 and FP16 population storage.
#include "ens_impl.cuh"

LBMAN_ENS_DEFINE(f32, float, float, true)
LBMAN_ENS_DEFINE(f16, float, __half, true)
