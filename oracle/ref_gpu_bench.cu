// ref_gpu_bench.cu -- times the reference's own FP64 CUDA solver: DeviceFields
// and DeviceSolver<SimBC> (src/cuda/device_fields.cu, src/cuda/device_solver.cu,
// src/cuda/kernels.cu), compiled from the reference's sources where they lie
// by oracle/build_ref.py, on this project's seeded initial condition.  TEST
// INFRASTRUCTURE ONLY: the GPU baseline the library's FP64 path is compared
// with.
//
// The call sequence is ActiveNematicSim's GPU path (src/active_nematic.h:
// 51-58, 85-86): LbmSolver::Initialize and the (injected) QTensorSolver
// initial Q on host fields, DeviceFields::Initialize, DeviceSolver::Initialize,
// then QTensorStep + LBMStep per step on the default stream, timed with CUDA
// events (Q stage and LBM separately).
//
// Usage: ref_gpu_bench <seed> <S0> <sigma> <warmup> <steps>
// Prints one JSON line.
#include <params.h>
#include <sim_config.h>

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <vector>

#include "device_fields.h"
#include "device_solver.h"
#include "fluid_fields.h"
#include "lbm_solver.h"
#include "lbman_oracle.h"
#include "qtensor_fields.h"

namespace {

void check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

}  // namespace

int main(int argc, char** argv) {
    try {
        if (argc != 6) throw std::runtime_error("usage: ref_gpu_bench <seed> <S0> <sigma> <warmup> <steps>");
        const uint64_t seed = std::strtoull(argv[1], nullptr, 10);
        const double S0 = std::atof(argv[2]), sigma = std::atof(argv[3]);
        const int warmup = std::atoi(argv[4]), steps = std::atoi(argv[5]);
        const LocalGrid g = LocalGrid::SingleRank();
        const int64_t V = static_cast<int64_t>(Params::nx) * Params::ny * Params::nz;

        FluidFields ff(g);
        QTensorFields qf(g);
        for (int64_t c = 0; c < V; ++c) {
            ff.rho[c] = 1.0;
            ff.ux[c] = ff.uy[c] = ff.uz[c] = 0.0;
        }
        LbmSolver<SimBC> lbm;
        lbm.Initialize(ff);
        {
            orc_params op;
            std::memset(&op, 0, sizeof(op));
            op.nx = Params::nx; op.ny = Params::ny; op.nz = Params::nz;
            std::vector<double> q(5 * V);
            orc_seeded_q(&op, seed, S0, sigma, q.data());
            double* comps[5] = {qf.qxx.data(), qf.qxy.data(), qf.qxz.data(), qf.qyy.data(), qf.qyz.data()};
            for (int k = 0; k < 5; ++k) std::memcpy(comps[k], q.data() + k * V, V * sizeof(double));
        }

        DeviceFields df(g);
        df.Initialize(ff, qf);
        DeviceSolver<SimBC> ds;
        ds.Initialize(df);
        for (int t = 0; t < warmup; ++t) {
            ds.QTensorStep(df);
            ds.LBMStep(df);
        }
        check(cudaDeviceSynchronize(), "warm-up");
        cudaEvent_t e0, e1, e2;
        check(cudaEventCreate(&e0), "event");
        check(cudaEventCreate(&e1), "event");
        check(cudaEventCreate(&e2), "event");
        double ms_q = 0.0, ms_l = 0.0;
        for (int t = 0; t < steps; ++t) {
            check(cudaEventRecord(e0), "record");
            ds.QTensorStep(df);
            check(cudaEventRecord(e1), "record");
            ds.LBMStep(df);
            check(cudaEventRecord(e2), "record");
            check(cudaEventSynchronize(e2), "step");
            float a = 0.f, b = 0.f;
            check(cudaEventElapsedTime(&a, e0, e1), "elapsed");
            check(cudaEventElapsedTime(&b, e1, e2), "elapsed");
            ms_q += a;
            ms_l += b;
        }
        // a finite-state check: the mass after the run
        std::vector<double> rho(V);
        check(cudaMemcpy(rho.data(), df.d_rho.data().get(), V * sizeof(double), cudaMemcpyDeviceToHost), "copy");
        double mass = 0.0;
        for (int64_t c = 0; c < V; ++c) mass += rho[c];
        std::printf("{\"steps\": %d, \"ms_q\": %.6f, \"ms_lbm\": %.6f, \"ms_step\": %.6f, \"mlups\": %.6f, "
                    "\"mass\": %.17g, \"cells\": %lld}\n",
                    steps, ms_q / steps, ms_l / steps, (ms_q + ms_l) / steps,
                    static_cast<double>(V) * steps / ((ms_q + ms_l) * 1e3), mass, static_cast<long long>(V));
        return 0;
    } catch (const std::exception& e) {
        std::printf("{\"error\": \"%s\"}\n", e.what());
        return 2;
    }
}
