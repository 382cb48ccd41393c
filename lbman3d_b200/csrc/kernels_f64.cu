// kernels_f64.cu -- FP64 instantiation (compute and storage in double).
// Built with --fmad=false: together with the association order kept in
// physics.cuh / lbm.cuh this makes the FP64 path bitwise equal to the
// reference CPU solver.
#include "kernels_impl.cuh"

LBMAN_DEFINE_LAUNCHERS(f64, double, double, false)

namespace lbman {
cudaError_t launch_fold(const double* partials, int G, int nq, int nmax, double* out, cudaStream_t st) {
    fold_partials_kernel<<<1, 1024, 0, st>>>(partials, G, nq, nmax, out);
    return cudaGetLastError();
}
}  // namespace lbman
