// solver_view.h -- in-library access to a single-box solver's device state
// for the closure code (closure_api.cu).  Not part of the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

struct lbman_solver;
struct lbman_ensemble;

namespace lbman {

struct SolverView {
    int prec;               // LBMAN_FP64 / LBMAN_FP32 / LBMAN_FP16
    int nx, ny, nz;
    int64_t V;
    void* rho;              // [V]   compute type (double for FP64, else float)
    void* u;                // [3V]
    void* q;                // [5V]
    cudaStream_t stream;
    bool uploaded;
};

int solver_view(lbman_solver* s, SolverView* v);
// The current fields of box `box` of an ensemble (rho is current after every
// lbman_ensemble_step call).
int ensemble_box_view(lbman_ensemble* e, int box, SolverView* v);
// Rebuild the populations as f_eq(rho, u) of the current fields (as after an
// upload without populations); the next step starts from them.
int solver_reset_populations(lbman_solver* s);
// Replace rho, u, Q by device fields of the solver's compute type (zero body
// force, f = f_eq).
int solver_set_state(lbman_solver* s, const void* rho, const void* u3, const void* q5);
void set_last_error(const char* msg);

}  // namespace lbman
