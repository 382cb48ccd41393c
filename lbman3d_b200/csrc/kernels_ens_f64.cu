// kernels_ens_f64.cu -- ensemble launchers for FP64 (built with --fmad=false).
#include "ens_impl.cuh"

LBMAN_ENS_DEFINE(f64, double, double, false)
