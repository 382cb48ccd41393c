// dropin_check.cc -- runs the reference's own CPU solver classes and the C++
// drop-in (include/lbman3d_dropin.hpp over liblbman3d_b200.so) side by side
// on the same fields and compares them bit for bit.  TEST INFRASTRUCTURE
// ONLY: built by oracle/build_ref.py against the reference sources where
// they lie, with a generated params.h/sim_config.h first on the include path
// (the shadowing of the reference's tests/CMakeLists.txt:3-8).
//
// Three call sequences are checked per boundary configuration:
//   sim   : ActiveNematicSim's GPU sequence (src/active_nematic.h:51-108):
//           LbmSolver::Initialize, DeviceFields::Initialize,
//           DeviceSolver::Initialize, then per step QTensorStep + LBMStep,
//           and DeviceFields::CopyToHost, against the CPU sequence
//           QTensorSolver::Step + LbmSolver::LatticeBoltzmannStep.
//   lbm   : lbman::LbmSolver<BC>::Initialize / LatticeBoltzmannStep on host
//           fields against LbmSolver<BC> (populations compared too).
//   q     : lbman::QTensorSolver<BC>::Step against QTensorSolver<BC>::Step
//           (new Q and the full body force compared).
//   q_setup : StepAndSetupBodyForce alone (new and previous Q, Sigma, tau,
//           Ericksen seed compared).
//   q_zero / q_varying / q_init_only : Step of subclasses written once and
//           derived from either class -- the empty override the reference
//           documents for pure relaxation (src/qtensor_solver.h:21), an
//           override that calls the base and adds a space-varying active
//           term (the VaryingAlpha pattern, src/qtensor_solver.h:11-19), and
//           a subclass that overrides only Initialize.
//
// Usage: dropin_check <steps>      prints one JSON line per check, exit 0
//                                  iff every field matched bitwise.
#include <params.h>
#include <sim_config.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numbers>
#include <string>
#include <vector>

#include "fluid_fields.h"
#include "lbm_solver.h"
#include "qtensor_fields.h"
#include "qtensor_solver.h"
#include "lbman3d_dropin.hpp"

namespace {

// The reference's SlitConfig (src/sim_config.h:19-27); the generated
// sim_config.h shadows the file that defines it.
struct SlitCfg {
    using XLo = WallSpec<Neumann, SpecularReflection>;
    using XHi = WallSpec<Neumann, SpecularReflection>;
    using YLo = WallSpec<Periodic, Periodic>;
    using YHi = WallSpec<Periodic, Periodic>;
    using ZLo = WallSpec<Periodic, Periodic>;
    using ZHi = WallSpec<Periodic, Periodic>;
    static constexpr std::string_view name = "Slit";
};
struct MixedCfg {
    using XLo = WallSpec<Neumann, SpecularReflection>;
    using XHi = WallSpec<Anchoring<0.5, 0.7, 1.1>, SpecularReflection>;
    using YLo = WallSpec<Periodic, Periodic>;
    using YHi = WallSpec<Periodic, Periodic>;
    using ZLo = WallSpec<Anchoring<0.3, 0.2, 0.5>, NoSlip>;
    using ZHi = WallSpec<Neumann, MovingWall<0.0, 0.02, 0.01>>;
    static constexpr std::string_view name = "Mixed";
};

// Deterministic test fields: a splitmix64 hash of (cell, component).
uint64_t mix(uint64_t z) {
    z += 0x9e3779b97f4a7c15ULL;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}
double unit(uint64_t cell, int k) { return (double)(mix(cell * 16 + k) >> 11) * 0x1.0p-53 - 0.5; }

void fill(FluidFields& ff, QTensorFields& qf) {
    const LocalGrid& g = ff.grid;
    const int64_t V = (int64_t)g.local_nx * g.local_ny * g.local_nz;
    for (int64_t c = 0; c < V; ++c) {
        ff.rho[c] = 1.0 + 0.02 * unit(c, 0);
        ff.ux[c] = 0.01 * unit(c, 1);
        ff.uy[c] = 0.01 * unit(c, 2);
        ff.uz[c] = 0.01 * unit(c, 3);
        ff.fx[c] = ff.fy[c] = ff.fz[c] = 0.0;
        qf.qxx[c] = -0.5 / 3.0 + 0.05 * unit(c, 4);
        qf.qxy[c] = 0.05 * unit(c, 5);
        qf.qxz[c] = 0.05 * unit(c, 6);
        qf.qyy[c] = -0.5 / 3.0 + 0.05 * unit(c, 7);
        qf.qyz[c] = 0.05 * unit(c, 8);
    }
}

// Subclasses of the reference's QTensorSolver and of the drop-in, from one
// source: Base is ::QTensorSolver<BC> or lbman::QTensorSolver<BC>.
template <class Base>
struct ZeroActivity : Base {
    void SetActiveStressAndComputeBodyForce(FluidFields&, const QTensorFields&) const override {}
};
template <class Base>
struct VaryingAlpha : Base {
    void SetActiveStressAndComputeBodyForce(FluidFields& ff, const QTensorFields& qf) const override {
        Base::SetActiveStressAndComputeBodyForce(ff, qf);
        const LocalGrid& g = qf.grid;
        const int nx = g.local_nx, ny = g.local_ny, nz = g.local_nz;
        for (int z = 0; z < nz; ++z)
            for (int y = 0; y < ny; ++y)
                for (int x = 0; x < nx; ++x) {
                    const int64_t c = ((int64_t)z * ny + y) * nx + x;
                    const int64_t xm = c - x + (x + nx - 1) % nx, xp = c - x + (x + 1) % nx;
                    const double a = 0.01 * std::sin(2.0 * std::numbers::pi * x / nx);
                    ff.fx[c] += -a * 0.5 * (qf.qxx[xp] - qf.qxx[xm]);
                    ff.fy[c] += -a * 0.5 * (qf.qxy[xp] - qf.qxy[xm]);
                    ff.fz[c] += -a * 0.5 * (qf.qxz[xp] - qf.qxz[xm]);
                }
    }
};
template <class Base>
struct InitOnly : Base {
    void Initialize(QTensorFields& qf) const override { Base::Initialize(qf); }
};

struct Cmp {
    int64_t mismatches = 0;
    double max_abs = 0.0;
    void add(const std::vector<double>& a, const std::vector<double>& b, int64_t n) {
        for (int64_t i = 0; i < n; ++i) {
            if (std::memcmp(&a[i], &b[i], sizeof(double)) != 0) {
                ++mismatches;
                const double d = std::fabs(a[i] - b[i]);
                if (!(d <= max_abs)) max_abs = d;
            }
        }
    }
};

void report(const char* check, std::string_view bc, int steps, const Cmp& c, bool& ok) {
    std::printf("{\"check\": \"%s\", \"bc\": \"%.*s\", \"steps\": %d, \"mismatches\": %lld, \"max_abs\": %.3e}\n",
                check, (int)bc.size(), bc.data(), steps, (long long)c.mismatches, c.max_abs);
    ok = ok && c.mismatches == 0;
}

template <typename BC>
void check_bc(int steps, bool& ok) {
    const LocalGrid g = LocalGrid::SingleRank();
    const int64_t V = (int64_t)g.local_nx * g.local_ny * g.local_nz;

    // sim: CPU reference sequence vs the drop-in device sequence.
    {
        FluidFields ffr(g), ffd(g);
        QTensorFields qfr(g), qfd(g);
        fill(ffr, qfr);
        fill(ffd, qfd);
        LbmSolver<BC> lbm;
        QTensorSolver<BC> qs;
        lbm.Initialize(ffr);
        lbm.Initialize(ffd);
        for (int n = 0; n < steps; ++n) {
            qs.Step(qfr, ffr);
            lbm.LatticeBoltzmannStep(ffr);
        }
        DeviceFields df(g);
        DeviceSolver<BC> ds;
        df.Initialize(ffd, qfd);
        ds.Initialize(df);
        for (int n = 0; n < steps; ++n) {
            ds.QTensorStep(df);
            ds.LBMStep(df);
        }
        df.CopyToHost(ffd, qfd);
        Cmp c;
        c.add(ffr.rho, ffd.rho, V);
        c.add(ffr.ux, ffd.ux, V);
        c.add(ffr.uy, ffd.uy, V);
        c.add(ffr.uz, ffd.uz, V);
        c.add(qfr.qxx, qfd.qxx, V);
        c.add(qfr.qxy, qfd.qxy, V);
        c.add(qfr.qxz, qfd.qxz, V);
        c.add(qfr.qyy, qfd.qyy, V);
        c.add(qfr.qyz, qfd.qyz, V);
        report("sim", BC::name, steps, c, ok);
    }
    // lbm: host-field LbmSolver.
    {
        FluidFields ffr(g), ffd(g);
        QTensorFields qfr(g), qfd(g);
        fill(ffr, qfr);
        fill(ffd, qfd);
        for (int64_t c = 0; c < V; ++c) {
            ffr.fx[c] = ffd.fx[c] = 1e-4 * unit(c, 9);
            ffr.fy[c] = ffd.fy[c] = 1e-4 * unit(c, 10);
            ffr.fz[c] = ffd.fz[c] = 1e-4 * unit(c, 11);
        }
        LbmSolver<BC> ref;
        lbman::LbmSolver<BC> gpu;
        ref.Initialize(ffr);
        gpu.Initialize(ffd);
        Cmp c0;
        c0.add(ffr.f, ffd.f, 15 * V);
        report("lbm_init", BC::name, 0, c0, ok);
        for (int n = 0; n < steps; ++n) {
            ref.LatticeBoltzmannStep(ffr);
            gpu.LatticeBoltzmannStep(ffd);
        }
        Cmp c;
        c.add(ffr.f, ffd.f, 15 * V);
        c.add(ffr.rho, ffd.rho, V);
        c.add(ffr.ux, ffd.ux, V);
        c.add(ffr.uy, ffd.uy, V);
        c.add(ffr.uz, ffd.uz, V);
        report("lbm", BC::name, steps, c, ok);
    }
    // q: host-field QTensorSolver::Step.
    {
        FluidFields ffr(g), ffd(g);
        QTensorFields qfr(g), qfd(g);
        fill(ffr, qfr);
        fill(ffd, qfd);
        QTensorSolver<BC> ref;
        lbman::QTensorSolver<BC> gpu;
        ref.Step(qfr, ffr);
        gpu.Step(qfd, ffd);
        Cmp c;
        c.add(qfr.qxx, qfd.qxx, V);
        c.add(qfr.qxy, qfd.qxy, V);
        c.add(qfr.qxz, qfd.qxz, V);
        c.add(qfr.qyy, qfd.qyy, V);
        c.add(qfr.qyz, qfd.qyz, V);
        c.add(ffr.fx, ffd.fx, V);
        c.add(ffr.fy, ffd.fy, V);
        c.add(ffr.fz, ffd.fz, V);
        report("q", BC::name, 1, c, ok);
    }
    // q_setup: phase 1 alone.
    {
        FluidFields ffr(g), ffd(g);
        QTensorFields qfr(g), qfd(g);
        fill(ffr, qfr);
        fill(ffd, qfd);
        QTensorSolver<BC> ref;
        lbman::QTensorSolver<BC> gpu;
        ref.StepAndSetupBodyForce(qfr, ffr);
        gpu.StepAndSetupBodyForce(qfd, ffd);
        Cmp c;
        c.add(qfr.qxx, qfd.qxx, V); c.add(qfr.qxy, qfd.qxy, V); c.add(qfr.qxz, qfd.qxz, V);
        c.add(qfr.qyy, qfd.qyy, V); c.add(qfr.qyz, qfd.qyz, V);
        c.add(qfr.qxx_new, qfd.qxx_new, V); c.add(qfr.qyz_new, qfd.qyz_new, V);
        c.add(qfr.Sigma_xx, qfd.Sigma_xx, V); c.add(qfr.Sigma_xy, qfd.Sigma_xy, V);
        c.add(qfr.Sigma_xz, qfd.Sigma_xz, V); c.add(qfr.Sigma_yy, qfd.Sigma_yy, V);
        c.add(qfr.Sigma_yz, qfd.Sigma_yz, V);
        c.add(qfr.Tau_xy, qfd.Tau_xy, V); c.add(qfr.Tau_xz, qfd.Tau_xz, V); c.add(qfr.Tau_yz, qfd.Tau_yz, V);
        c.add(ffr.fx, ffd.fx, V); c.add(ffr.fy, ffd.fy, V); c.add(ffr.fz, ffd.fz, V);
        report("q_setup", BC::name, 1, c, ok);
    }
    // Subclasses: Step of each, two steps in a row.
    auto sub = [&](const char* name, const auto& ref, const auto& gpu) {
        FluidFields ffr(g), ffd(g);
        QTensorFields qfr(g), qfd(g);
        fill(ffr, qfr);
        fill(ffd, qfd);
        for (int n = 0; n < 2; ++n) {
            ref.Step(qfr, ffr);
            gpu.Step(qfd, ffd);
        }
        Cmp c;
        c.add(qfr.qxx, qfd.qxx, V); c.add(qfr.qxy, qfd.qxy, V); c.add(qfr.qxz, qfd.qxz, V);
        c.add(qfr.qyy, qfd.qyy, V); c.add(qfr.qyz, qfd.qyz, V);
        c.add(ffr.fx, ffd.fx, V); c.add(ffr.fy, ffd.fy, V); c.add(ffr.fz, ffd.fz, V);
        report(name, BC::name, 2, c, ok);
    };
    sub("q_zero", ZeroActivity<QTensorSolver<BC>>{}, ZeroActivity<lbman::QTensorSolver<BC>>{});
    sub("q_varying", VaryingAlpha<QTensorSolver<BC>>{}, VaryingAlpha<lbman::QTensorSolver<BC>>{});
    sub("q_init_only", InitOnly<QTensorSolver<BC>>{}, InitOnly<lbman::QTensorSolver<BC>>{});
}

}  // namespace

int main(int argc, char** argv) {
    const int steps = argc > 1 ? std::atoi(argv[1]) : 5;
    bool ok = true;
    try {
        check_bc<FullyPeriodicConfig>(steps, ok);
        check_bc<SlitCfg>(steps, ok);
        check_bc<ChannelConfig>(steps, ok);
        check_bc<MixedCfg>(steps, ok);
    } catch (const std::exception& e) {
        std::printf("{\"error\": \"%s\"}\n", e.what());
        return 2;
    }
    return ok ? 0 : 1;
}
