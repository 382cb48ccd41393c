// ref_driver.cc -- runs the reference's own CPU solver classes on a field
// file and writes the resulting fields.  TEST INFRASTRUCTURE ONLY.
//
// Built by oracle/build_ref.py against the reference sources where they lie
// (src/lbm_solver.h, src/qtensor_solver.h, src/analysis_fields.h,
// src/analysis/defect_finder.h plus src/fluid_fields.cc,
// src/qtensor_fields.cc, src/analysis_fields.cc,
// src/analysis/defect_fields.cc), with a generated params.h/sim_config.h
// first on the include path -- the same shadowing the reference's own tests
// use (tests/CMakeLists.txt:3-8).  Outputs go to oracle/_ref/ only.
//
// The step sequence is the reference CPU path of ActiveNematicSim::Step
// (src/active_nematic.h:84-108) as driven by its integration fixtures
// (tests/integration/test_coupled_backflow.cc:117-126): QTensorSolver::Step,
// then LbmSolver::LatticeBoltzmannStep.  Initial fields are injected the way
// the reference tests do it, by overriding QTensorSolver::Initialize
// (tests/integration/test_coupled_backflow.cc:67-86).
//
// Usage:
//   ref_driver <bc> <mode> <in.bin> <out.bin> <snap1> [snap2 ...]
//   ref_driver --bench <bc> <seed> <S0> <sigma> <warmup> <steps>
// mode: full | q | q_active | lbm
// in.bin : int64 V, int32 has_f, int32 has_force, rho[V] u[3V] q[5V]
//          [f[15V] direction-major] [force[3V]]   (float64, little endian)
// out.bin: per snapshot: int64 step, rho, u(3), q(5), f(15, direction-major),
//          force(3), sigma(5), tau(3), order, director(3, AoS), then
//          float64 {free_energy, mass, px, py, pz, ke, e1, e2, umax2},
//          int64 defect_face_count, int64 disclinations.
#include <params.h>
#include <sim_config.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <memory>
#include <numbers>
#include <stdexcept>
#include <string>
#include <vector>

#include "analysis/defect_finder.h"
#include "lbman_oracle.h"
#include "analysis_fields.h"
#include "fluid_fields.h"
#include "lbm_solver.h"
#include "qtensor_fields.h"
#include "qtensor_solver.h"

using namespace Params;

// Boundary configurations exercised by the parity suite.  The first four are
// the reference presets (src/boundary.h:105-129, src/sim_config.h:19-45);
// the rest are the custom configurations of its integration tests
// (tests/integration/test_bc_combinations.cc:182-227,
// tests/integration/test_poiseuille.cc:88-96) and combinations that drive
// every wall rule at edges and corners.
struct SlitCfg {
    using XLo = WallSpec<Neumann, SpecularReflection>;
    using XHi = WallSpec<Neumann, SpecularReflection>;
    using YLo = WallSpec<Periodic, Periodic>;
    using YHi = WallSpec<Periodic, Periodic>;
    using ZLo = WallSpec<Periodic, Periodic>;
    using ZHi = WallSpec<Periodic, Periodic>;
    static constexpr std::string_view name = "SlitFreeSlip";
};
struct SlitNoSlipCfg {
    using XLo = WallSpec<Neumann, NoSlip>;
    using XHi = WallSpec<Neumann, NoSlip>;
    using YLo = WallSpec<Periodic, Periodic>;
    using YHi = WallSpec<Periodic, Periodic>;
    using ZLo = WallSpec<Periodic, Periodic>;
    using ZHi = WallSpec<Periodic, Periodic>;
    static constexpr std::string_view name = "SlitNoSlip";
};
struct PoiseuilleCfg {
    using XLo = WallSpec<Periodic, Periodic>;
    using XHi = WallSpec<Periodic, Periodic>;
    using YLo = WallSpec<Neumann, NoSlip>;
    using YHi = WallSpec<Neumann, NoSlip>;
    using ZLo = WallSpec<Periodic, Periodic>;
    using ZHi = WallSpec<Periodic, Periodic>;
    static constexpr std::string_view name = "Poiseuille";
};
struct SpecularZCfg {
    using XLo = WallSpec<Periodic, Periodic>;
    using XHi = WallSpec<Periodic, Periodic>;
    using YLo = WallSpec<Periodic, Periodic>;
    using YHi = WallSpec<Periodic, Periodic>;
    using ZLo = WallSpec<Neumann, SpecularReflection>;
    using ZHi = WallSpec<Neumann, SpecularReflection>;
    static constexpr std::string_view name = "SpecularZ";
};
struct AnchoredZCfg {
    using XLo = WallSpec<Periodic, Periodic>;
    using XHi = WallSpec<Periodic, Periodic>;
    using YLo = WallSpec<Periodic, Periodic>;
    using YHi = WallSpec<Periodic, Periodic>;
    using ZLo = WallSpec<Anchoring<0.5, std::numbers::pi / 4.0, 0.0>, NoSlip>;
    using ZHi = WallSpec<Anchoring<0.5, std::numbers::pi / 4.0, 0.0>, NoSlip>;
    static constexpr std::string_view name = "AnchoredZ";
};
struct LidCfg {
    using XLo = WallSpec<Periodic, Periodic>;
    using XHi = WallSpec<Periodic, Periodic>;
    using YLo = WallSpec<Neumann, NoSlip>;
    using YHi = WallSpec<Anchoring<0.4, 1.0, 0.3>, MovingWall<0.05, 0.0, 0.02>>;
    using ZLo = WallSpec<Periodic, Periodic>;
    using ZHi = WallSpec<Periodic, Periodic>;
    static constexpr std::string_view name = "Lid";
};
struct BoxMixedCfg {
    using XLo = WallSpec<Neumann, SpecularReflection>;
    using XHi = WallSpec<Anchoring<0.5, 0.7, 1.1>, SpecularReflection>;
    using YLo = WallSpec<Neumann, NoSlip>;
    using YHi = WallSpec<Neumann, MovingWall<0.03, 0.0, -0.01>>;
    using ZLo = WallSpec<Anchoring<0.3, 0.2, 0.5>, NoSlip>;
    using ZHi = WallSpec<Neumann, MovingWall<0.0, 0.02, 0.0>>;
    static constexpr std::string_view name = "BoxMixed";
};
struct QMixedCfg {
    using XLo = WallSpec<Periodic, Periodic>;
    using XHi = WallSpec<Neumann, Periodic>;
    using YLo = WallSpec<Anchoring<0.5, 0.3, 0.2>, Periodic>;
    using YHi = WallSpec<Anchoring<0.5, 0.3, 0.2>, Periodic>;
    using ZLo = WallSpec<Neumann, SpecularReflection>;
    using ZHi = WallSpec<Neumann, NoSlip>;
    static constexpr std::string_view name = "QMixed";
};
using AllWallsCfg = BCConfig<>;

namespace {

std::vector<double> g_rho, g_u, g_q, g_f, g_force;
bool g_has_f = false, g_has_force = false;
int64_t g_V = 0;

// Injects the fields read from in.bin, the subclass-override pattern of the
// reference tests.
template <typename BC, bool Active>
class InjectedSolver : public QTensorSolver<BC> {
public:
    void Initialize(QTensorFields& qf) const override {
        double* comps[5] = {qf.qxx.data(), qf.qxy.data(), qf.qxz.data(), qf.qyy.data(), qf.qyz.data()};
        for (int k = 0; k < 5; ++k)
            for (int64_t c = 0; c < g_V; ++c) comps[k][c] = g_q[k * g_V + c];
    }
    void SetActiveStressAndComputeBodyForce(FluidFields& ff, const QTensorFields& qf) const override {
        if constexpr (Active) QTensorSolver<BC>::SetActiveStressAndComputeBodyForce(ff, qf);
    }
};

void put(FILE* fp, const double* v, size_t n) {
    if (std::fwrite(v, sizeof(double), n, fp) != n) throw std::runtime_error("write failed");
}

template <typename BC>
void write_snapshot(FILE* fp, int64_t step, const FluidFields& ff, const QTensorFields& qf,
                    std::vector<double>& upast) {
    const int64_t V = g_V;
    put(fp, reinterpret_cast<const double*>(&step), 1);
    put(fp, ff.rho.data(), V);
    put(fp, ff.ux.data(), V); put(fp, ff.uy.data(), V); put(fp, ff.uz.data(), V);
    put(fp, qf.qxx.data(), V); put(fp, qf.qxy.data(), V); put(fp, qf.qxz.data(), V);
    put(fp, qf.qyy.data(), V); put(fp, qf.qyz.data(), V);
    std::vector<double> soa(15 * V);
    for (int64_t c = 0; c < V; ++c)
        for (int i = 0; i < 15; ++i) soa[i * V + c] = ff.f[c * 15 + i];
    put(fp, soa.data(), 15 * V);
    put(fp, ff.fx.data(), V); put(fp, ff.fy.data(), V); put(fp, ff.fz.data(), V);
    put(fp, qf.Sigma_xx.data(), V); put(fp, qf.Sigma_xy.data(), V); put(fp, qf.Sigma_xz.data(), V);
    put(fp, qf.Sigma_yy.data(), V); put(fp, qf.Sigma_yz.data(), V);
    put(fp, qf.Tau_xy.data(), V); put(fp, qf.Tau_xz.data(), V); put(fp, qf.Tau_yz.data(), V);

    AnalysisFields af(ff.grid);
    QtensorToOrderDirector(qf, af);
    put(fp, af.order_.data(), V);
    put(fp, af.director_.data(), 3 * V);

    // SimIO::Log's reductions (src/sim_io.cc:83-108), same accumulation order.
    double mass = 0, px = 0, py = 0, pz = 0, ke = 0, e1 = 0, e2 = 0, umax2 = 0;
    for (int64_t c = 0; c < V; ++c) {
        mass += ff.rho[c];
        px += ff.rho[c] * ff.ux[c];
        py += ff.rho[c] * ff.uy[c];
        pz += ff.rho[c] * ff.uz[c];
        const double u2 = ff.ux[c] * ff.ux[c] + ff.uy[c] * ff.uy[c] + ff.uz[c] * ff.uz[c];
        ke += 0.5 * ff.rho[c] * u2;
        if (u2 > umax2) umax2 = u2;
        e1 += (ff.ux[c] - upast[c]) * (ff.ux[c] - upast[c]) +
              (ff.uy[c] - upast[V + c]) * (ff.uy[c] - upast[V + c]) +
              (ff.uz[c] - upast[2 * V + c]) * (ff.uz[c] - upast[2 * V + c]);
        e2 += u2;
        upast[c] = ff.ux[c]; upast[V + c] = ff.uy[c]; upast[2 * V + c] = ff.uz[c];
    }
    const double fe = TotalNematicFreeEnergy<BC>(qf);
    const double diag[9] = {fe, mass, px, py, pz, ke, e1, e2, umax2};
    put(fp, diag, 9);

    // The defect graph code indexes face arrays that are empty when an axis
    // has a single cell, so grids thinner than 2 cells report -1.
    int64_t nflag = -1, ndisc = -1;
    if (nx >= 2 && ny >= 2 && nz >= 2) {
        DefectFields df;
        DefectFinder<BC> finder;
        finder.FindDefects(af, df);
        nflag = 0;
        for (auto v : df.def_x) nflag += v;
        for (auto v : df.def_y) nflag += v;
        for (auto v : df.def_z) nflag += v;
        ndisc = static_cast<int64_t>(df.disclinations.size());
    }
    std::fwrite(&nflag, sizeof(int64_t), 1, fp);
    std::fwrite(&ndisc, sizeof(int64_t), 1, fp);
}

template <typename BC>
int run(const std::string& mode, const char* in_path, const char* out_path,
        const std::vector<int64_t>& snaps) {
    FILE* fin = std::fopen(in_path, "rb");
    if (!fin) throw std::runtime_error("cannot open input");
    int64_t V = 0; int32_t hf = 0, hF = 0;
    if (std::fread(&V, 8, 1, fin) != 1 || std::fread(&hf, 4, 1, fin) != 1 || std::fread(&hF, 4, 1, fin) != 1)
        throw std::runtime_error("bad header");
    if (V != static_cast<int64_t>(nx) * ny * nz) throw std::runtime_error("grid size mismatch with params.h");
    g_V = V; g_has_f = hf != 0; g_has_force = hF != 0;
    auto get = [&](std::vector<double>& v, size_t n) {
        v.resize(n);
        if (std::fread(v.data(), sizeof(double), n, fin) != n) throw std::runtime_error("short input");
    };
    get(g_rho, V); get(g_u, 3 * V); get(g_q, 5 * V);
    if (g_has_f) get(g_f, 15 * V);
    if (g_has_force) get(g_force, 3 * V);
    std::fclose(fin);

    LocalGrid grid = LocalGrid::SingleRank();
    FluidFields ff(grid);
    QTensorFields qf(grid);
    LbmSolver<BC> lbm;
    std::unique_ptr<QTensorSolver<BC>> qs;
    if (mode == "q") qs = std::make_unique<InjectedSolver<BC, false>>();
    else qs = std::make_unique<InjectedSolver<BC, true>>();

    for (int64_t c = 0; c < V; ++c) {
        ff.rho[c] = g_rho[c]; ff.ux[c] = g_u[c]; ff.uy[c] = g_u[V + c]; ff.uz[c] = g_u[2 * V + c];
        if (g_has_force) { ff.fx[c] = g_force[c]; ff.fy[c] = g_force[V + c]; ff.fz[c] = g_force[2 * V + c]; }
    }
    if (g_has_f) {
        for (int64_t c = 0; c < V; ++c)
            for (int i = 0; i < 15; ++i) ff.f[c * 15 + i] = g_f[i * V + c];
    } else {
        lbm.Initialize(ff);
    }
    qs->Initialize(qf);

    FILE* fout = std::fopen(out_path, "wb");
    if (!fout) throw std::runtime_error("cannot open output");
    std::vector<double> upast(3 * V, 0.0);
    int64_t done = 0;
    for (int64_t target : snaps) {
        for (; done < target; ++done) {
            if (mode == "full") { qs->Step(qf, ff); lbm.LatticeBoltzmannStep(ff); }
            else if (mode == "q" || mode == "q_active") qs->Step(qf, ff);
            else if (mode == "lbm") lbm.LatticeBoltzmannStep(ff);
            else throw std::runtime_error("unknown mode");
        }
        write_snapshot<BC>(fout, done, ff, qf, upast);
    }
    std::fclose(fout);
    return 0;
}

// Timing loop of src/benchmark.cc:21-50 (std::chrono around each full step),
// on the project's seeded initial condition (rho = 1, u = 0, Q from
// orc_seeded_q of oracle/lbman_oracle.c, the generator every workload of this
// project uses), generated in-process so large boxes need no input file.
template <typename BC>
int bench(uint64_t seed, double S0, double sigma, int warmup, int steps) {
    const int64_t V = static_cast<int64_t>(nx) * ny * nz;
    g_V = V;
    {
        orc_params op;
        std::memset(&op, 0, sizeof(op));
        op.nx = nx; op.ny = ny; op.nz = nz;
        g_q.resize(5 * V);
        orc_seeded_q(&op, seed, S0, sigma, g_q.data());
    }
    LocalGrid grid = LocalGrid::SingleRank();
    FluidFields ff(grid);
    QTensorFields qf(grid);
    LbmSolver<BC> lbm;
    InjectedSolver<BC, true> qs;
    for (int64_t c = 0; c < V; ++c) {
        ff.rho[c] = 1.0; ff.ux[c] = 0.0; ff.uy[c] = 0.0; ff.uz[c] = 0.0;
    }
    lbm.Initialize(ff);
    qs.Initialize(qf);
    std::vector<double>().swap(g_q);  // the solver holds its own copy now
    using clock = std::chrono::high_resolution_clock;
    for (int t = 0; t < warmup; ++t) { qs.Step(qf, ff); lbm.LatticeBoltzmannStep(ff); }
    double ms_q = 0, ms_l = 0;
    for (int t = 0; t < steps; ++t) {
        auto t0 = clock::now();
        qs.Step(qf, ff);
        auto t1 = clock::now();
        lbm.LatticeBoltzmannStep(ff);
        auto t2 = clock::now();
        ms_q += std::chrono::duration<double, std::milli>(t1 - t0).count();
        ms_l += std::chrono::duration<double, std::milli>(t2 - t1).count();
    }
    std::printf("{\"steps\": %d, \"threads\": %d, \"ms_q\": %.6f, \"ms_lbm\": %.6f, \"ms_step\": %.6f, "
                "\"mlups\": %.6f, \"rho0\": %.17g}\n",
                steps, static_cast<int>(kNumOMPThreads), ms_q / steps, ms_l / steps, (ms_q + ms_l) / steps,
                static_cast<double>(V) * steps / ((ms_q + ms_l) * 1e3), ff.rho[0]);
    return 0;
}

template <typename F>
int dispatch(const std::string& bc, F&& f) {
    if (bc == "periodic") return f.template operator()<FullyPeriodicConfig>();
    if (bc == "channel") return f.template operator()<ChannelConfig>();
    if (bc == "slit") return f.template operator()<SlitCfg>();
    if (bc == "slit_noslip") return f.template operator()<SlitNoSlipCfg>();
    if (bc == "poiseuille") return f.template operator()<PoiseuilleCfg>();
    if (bc == "specular_z") return f.template operator()<SpecularZCfg>();
    if (bc == "anchored_z") return f.template operator()<AnchoredZCfg>();
    if (bc == "lid") return f.template operator()<LidCfg>();
    if (bc == "box_mixed") return f.template operator()<BoxMixedCfg>();
    if (bc == "qmixed") return f.template operator()<QMixedCfg>();
    if (bc == "walls") return f.template operator()<AllWallsCfg>();
    throw std::runtime_error("unknown bc " + bc);
}

}  // namespace

int main(int argc, char** argv) {
    try {
        if (argc >= 2 && std::string(argv[1]) == "--bench") {
            if (argc != 8) throw std::runtime_error("usage: --bench <bc> <seed> <S0> <sigma> <warmup> <steps>");
            const uint64_t seed = std::strtoull(argv[3], nullptr, 10);
            const double S0 = std::atof(argv[4]), sigma = std::atof(argv[5]);
            const int w = std::atoi(argv[6]), s = std::atoi(argv[7]);
            return dispatch(argv[2], [&]<typename BC>() { return bench<BC>(seed, S0, sigma, w, s); });
        }
        if (argc < 6) throw std::runtime_error("usage: ref_driver <bc> <mode> <in.bin> <out.bin> <snap>...");
        std::vector<int64_t> snaps;
        for (int k = 5; k < argc; ++k) snaps.push_back(std::atoll(argv[k]));
        const std::string mode = argv[2];
        return dispatch(argv[1], [&]<typename BC>() { return run<BC>(mode, argv[3], argv[4], snaps); });
    } catch (const std::exception& e) {
        std::fprintf(stderr, "ref_driver: %s\n", e.what());
        return 2;
    }
}
