// lbman3d_dropin.hpp -- the reference's GPU-side interface over the C ABI of
// liblbman3d_b200.so (include/lbman3d.h).
//
// Include this instead of the reference's src/device_fields.h and
// src/device_solver.h (with the reference's src/ and the project's
// params.h / sim_config.h on the include path) and link
// liblbman3d_b200.so.  It provides, with the reference's signatures:
//
//   std::string InitializeComputeBackend(...)       src/device_fields.h:21
//   struct DeviceFields { DeviceFields(LocalGrid); Initialize(FluidFields&,
//       const QTensorFields&); CopyToHost(FluidFields&, QTensorFields&) const; }
//                                                    src/device_fields.h:23-56
//   template <class BC> struct DeviceSolver { Initialize(DeviceFields&);
//       QTensorStep(DeviceFields&); LBMStep(DeviceFields&); }
//                                                    src/device_solver.h:10-17
//   and GPU-backed lbman::LbmSolver<BC> / lbman::QTensorSolver<BC> with the
//   reference's CPU-solver signatures (src/lbm_solver.h:12-21,
//   src/qtensor_solver.h:23-52) operating on host fields.
//
// The reference's compile-time configuration is lowered here: Params::*
// (params.h) become lbman_config fields of the same names, the BC type's six
// WallSpec<QBC, UBC> become lbman_face descriptors, kQAdvection selects the
// advection scheme.  Non-zero statuses throw std::runtime_error, as the
// reference's checkCudaErrors does (src/cuda/cuda_utils.h:5-10).  Precision
// is FP64 (bitwise the reference's CPU arithmetic) unless
// LBMAN_DROPIN_PRECISION is defined to LBMAN_FP32 or LBMAN_FP16.
#pragma once

#include <params.h>
#include <sim_config.h>

#include <cmath>
#include <random>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <typeinfo>
#include <vector>

#include "boundary.h"
#include "fluid_fields.h"
#include "lbman3d.h"
#include "local_grid.h"
#include "qtensor_fields.h"

#ifndef LBMAN_DROPIN_PRECISION
#define LBMAN_DROPIN_PRECISION LBMAN_FP64
#endif

namespace lbman_dropin {

inline void check(int st) {
    if (st != LBMAN_OK)
        throw std::runtime_error(std::string("lbman: ") + lbman_status_string(st) + ": " + lbman_last_error());
}

template <typename QBC>
void lower_q(lbman_face& f) {
    if constexpr (std::is_same_v<QBC, Periodic>) {
        f.qbc = LBMAN_Q_PERIODIC;
    } else if constexpr (is_anchoring_v<QBC>) {
        f.qbc = LBMAN_Q_ANCHORING;
        f.s = QBC::s;
        f.theta = QBC::theta;
        f.phi = QBC::phi;
    } else {
        f.qbc = LBMAN_Q_NEUMANN;
    }
}

template <typename UBC>
void lower_u(lbman_face& f) {
    if constexpr (std::is_same_v<UBC, Periodic>) {
        f.ubc = LBMAN_U_PERIODIC;
    } else if constexpr (std::is_same_v<UBC, SpecularReflection>) {
        f.ubc = LBMAN_U_SPECULAR;
    } else if constexpr (is_moving_wall_v<UBC>) {
        f.ubc = LBMAN_U_MOVING;
        f.uw[0] = UBC::Ux;
        f.uw[1] = UBC::Uy;
        f.uw[2] = UBC::Uz;
    } else {
        f.ubc = LBMAN_U_NOSLIP;
    }
}

template <typename WS>
lbman_face lower_wall() {
    lbman_face f{};
    lower_q<typename WS::QBC>(f);
    lower_u<typename WS::UBC>(f);
    return f;
}

// params.h + BC type + sim_config.h -> lbman_config.
template <typename BC>
lbman_config make_config(const LocalGrid& g) {
    lbman_config c;
    check(lbman_config_init(&c));
    c.nx = g.local_nx;
    c.ny = g.local_ny;
    c.nz = g.local_nz;
    c.DT = Params::DT;
    c.kDensity = Params::kDensity;
    c.TAUF = Params::TAUF;
    c.L = Params::L;
    c.A = Params::A;
    c.B = Params::B;
    c.C = Params::C;
    c.LAMBDA = Params::LAMBDA;
    c.GAMMA = Params::GAMMA;
    c.ALPHA = Params::ALPHA;
    c.MU = Params::MU;
    c.advection = kQAdvection == Advection::Upwind ? LBMAN_UPWIND : LBMAN_CENTRED;
    c.face[0] = lower_wall<typename BC::XLo>();
    c.face[1] = lower_wall<typename BC::XHi>();
    c.face[2] = lower_wall<typename BC::YLo>();
    c.face[3] = lower_wall<typename BC::YHi>();
    c.face[4] = lower_wall<typename BC::ZLo>();
    c.face[5] = lower_wall<typename BC::ZHi>();
    c.precision = LBMAN_DROPIN_PRECISION;
    return c;
}

// Host-field marshalling between the reference's containers and the C ABI
// layout (populations AoS on the host, direction-major in the ABI).
struct Staging {
    std::vector<double> u3, q5, f15, F3;
    void from_fields(const FluidFields& ff, const QTensorFields& qf, int64_t V) {
        u3.resize(3 * V);
        q5.resize(5 * V);
        f15.resize(15 * V);
        F3.resize(3 * V);
        for (int64_t c = 0; c < V; ++c) {
            u3[c] = ff.ux[c]; u3[V + c] = ff.uy[c]; u3[2 * V + c] = ff.uz[c];
            F3[c] = ff.fx[c]; F3[V + c] = ff.fy[c]; F3[2 * V + c] = ff.fz[c];
            q5[c] = qf.qxx[c]; q5[V + c] = qf.qxy[c]; q5[2 * V + c] = qf.qxz[c];
            q5[3 * V + c] = qf.qyy[c]; q5[4 * V + c] = qf.qyz[c];
            for (int i = 0; i < 15; ++i) f15[i * V + c] = ff.f[c * 15 + i];
        }
    }
};

}  // namespace lbman_dropin

// Device description (src/device_fields.h:21).
template <typename... Ignored>
std::string InitializeComputeBackend(const Ignored&...) {
    char buf[2048];
    lbman_dropin::check(lbman_device_info(0, buf, sizeof(buf)));
    return buf;
}

// Device-resident fields (src/device_fields.h:23-56).  The solver handle is
// created by DeviceSolver<BC>::Initialize, which knows the BC type; the host
// fields handed to Initialize are uploaded then (the reference's
// ActiveNematicSim calls DeviceFields::Initialize immediately before
// DeviceSolver::Initialize, src/active_nematic.h:51-58).
struct DeviceFields {
    LocalGrid grid;
    lbman_solver* solver = nullptr;
    lbman_dropin::Staging pending;
    std::vector<double> pending_rho;
    bool has_pending = false;

    explicit DeviceFields(LocalGrid g = LocalGrid::SingleRank()) : grid(g) {
        // One rank owns the whole box; halo-padded MPI sub-domains are not
        // part of this boundary (host layout cell*15+i needs kHaloMPI == 0).
        if (g.kHaloMPI != 0) throw std::runtime_error("lbman: DeviceFields needs a single-rank LocalGrid (kHaloMPI == 0)");
    }
    DeviceFields(const DeviceFields&) = delete;
    DeviceFields& operator=(const DeviceFields&) = delete;
    ~DeviceFields() { lbman_destroy(solver); }

    int64_t V() const { return (int64_t)grid.local_nx * grid.local_ny * grid.local_nz; }

    void Initialize(FluidFields& ff, const QTensorFields& qf) {
        pending.from_fields(ff, qf, V());
        pending_rho.assign(ff.rho.begin(), ff.rho.begin() + V());
        has_pending = true;
        if (solver) upload_pending();
    }

    void upload_pending() {
        lbman_dropin::check(lbman_upload(solver, pending_rho.data(), pending.u3.data(), pending.q5.data(),
                                         pending.f15.data(), pending.F3.data()));
        has_pending = false;
    }

    void CopyToHost(FluidFields& ff, QTensorFields& qf) const {
        const int64_t V = this->V();
        std::vector<double> u3(3 * V), q5(5 * V);
        lbman_dropin::check(lbman_download(solver, ff.rho.data(), u3.data(), q5.data(), nullptr, nullptr));
        for (int64_t c = 0; c < V; ++c) {
            ff.ux[c] = u3[c]; ff.uy[c] = u3[V + c]; ff.uz[c] = u3[2 * V + c];
            qf.qxx[c] = q5[c]; qf.qxy[c] = q5[V + c]; qf.qxz[c] = q5[2 * V + c];
            qf.qyy[c] = q5[3 * V + c]; qf.qyz[c] = q5[4 * V + c];
        }
    }
};

// DeviceSolver<BC> (src/device_solver.h:10-17).
template <typename BC>
struct DeviceSolver {
    void Initialize(DeviceFields& df) {
        if (!df.solver) {
            const lbman_config cfg = lbman_dropin::make_config<BC>(df.grid);
            lbman_dropin::check(lbman_create(&cfg, &df.solver));
        }
        if (df.has_pending) df.upload_pending();
    }
    void QTensorStep(DeviceFields& df) { lbman_dropin::check(lbman_qtensor_step(df.solver)); }
    void LBMStep(DeviceFields& df) { lbman_dropin::check(lbman_lbm_step(df.solver)); }
};

namespace lbman {

// GPU-backed LbmSolver<BC> with the reference's signatures
// (src/lbm_solver.h:12-21): each call uploads the host fields, runs on the
// GPU and writes the results back (ff.f holds the new populations, as after
// the reference's SwapFandFnew).
template <typename BC>
class LbmSolver {
    mutable lbman_solver* s_ = nullptr;
    lbman_solver* get(const LocalGrid& g) const {
        if (!s_) {
            lbman_config cfg = lbman_dropin::make_config<BC>(g);
            cfg.kernels = LBMAN_KERNELS_SPLIT;
            lbman_dropin::check(lbman_create(&cfg, &s_));
        }
        return s_;
    }

public:
    LbmSolver() = default;
    LbmSolver(const LbmSolver&) = delete;
    ~LbmSolver() { lbman_destroy(s_); }

    void Initialize(FluidFields& ff) const {
        const LocalGrid& g = ff.grid;
        const int64_t V = (int64_t)g.local_nx * g.local_ny * g.local_nz;
        std::vector<double> u3(3 * V), q5(5 * V, 0.0), f15(15 * V);
        for (int64_t c = 0; c < V; ++c) { u3[c] = ff.ux[c]; u3[V + c] = ff.uy[c]; u3[2 * V + c] = ff.uz[c]; }
        lbman_solver* s = get(g);
        lbman_dropin::check(lbman_upload(s, ff.rho.data(), u3.data(), q5.data(), nullptr, nullptr));
        lbman_dropin::check(lbman_download(s, nullptr, nullptr, nullptr, f15.data(), nullptr));
        for (int64_t c = 0; c < V; ++c)
            for (int i = 0; i < 15; ++i) ff.f[c * 15 + i] = f15[i * V + c];
    }

    void LatticeBoltzmannStep(FluidFields& ff) const {
        const LocalGrid& g = ff.grid;
        const int64_t V = (int64_t)g.local_nx * g.local_ny * g.local_nz;
        QTensorFields dummy(g);
        lbman_dropin::Staging st;
        st.from_fields(ff, dummy, V);
        lbman_solver* s = get(g);
        lbman_dropin::check(lbman_upload(s, ff.rho.data(), st.u3.data(), st.q5.data(), st.f15.data(), st.F3.data()));
        lbman_dropin::check(lbman_lbm_step(s));
        std::vector<double> u3(3 * V);
        lbman_dropin::check(lbman_download(s, ff.rho.data(), u3.data(), nullptr, st.f15.data(), nullptr));
        for (int64_t c = 0; c < V; ++c) {
            ff.ux[c] = u3[c]; ff.uy[c] = u3[V + c]; ff.uz[c] = u3[2 * V + c];
            for (int i = 0; i < 15; ++i) ff.f[c * 15 + i] = st.f15[i * V + c];
        }
    }
};

// GPU-backed QTensorSolver<BC> (src/qtensor_solver.h:23-52) with the
// reference's two-phase contract: StepAndSetupBodyForce writes Q_new (after
// the swap of src/qtensor_solver.tpp:150-152), Sigma, tau and the Ericksen
// seed of the body force to the host fields; the virtual
// SetActiveStressAndComputeBodyForce then adds the active, passive and
// friction terms, and a subclass override replaces it as in the reference
// (src/qtensor_solver.h:11-21).  Step runs the two phases, except for an
// object of exactly this class (no subclass, so no override), where one GPU
// pass computes the same Q and force; that pass does not refresh
// qf.Sigma_* / qf.Tau_*, which nothing but the second phase reads.
template <typename BC>
class QTensorSolver {
    mutable lbman_solver* s_ = nullptr;

    lbman_solver* get(const LocalGrid& g) const {
        if (!s_) {
            lbman_config cfg = lbman_dropin::make_config<BC>(g);
            cfg.kernels = LBMAN_KERNELS_SPLIT;
            lbman_dropin::check(lbman_create(&cfg, &s_));
        }
        return s_;
    }
    static int64_t volume(const LocalGrid& g) { return (int64_t)g.local_nx * g.local_ny * g.local_nz; }

    // new Q (q5) into qf, the previous Q into qf.*_new, as SwapWithNew leaves them
    static void store_q(QTensorFields& qf, const std::vector<double>& q5, int64_t V) {
        std::vector<double>* cur[5] = {&qf.qxx, &qf.qxy, &qf.qxz, &qf.qyy, &qf.qyz};
        std::vector<double>* old[5] = {&qf.qxx_new, &qf.qxy_new, &qf.qxz_new, &qf.qyy_new, &qf.qyz_new};
        for (int k = 0; k < 5; ++k)
            for (int64_t c = 0; c < V; ++c) {
                (*old[k])[c] = (*cur[k])[c];
                (*cur[k])[c] = q5[k * V + c];
            }
    }
    static void store_force(FluidFields& ff, const std::vector<double>& F3, int64_t V) {
        for (int64_t c = 0; c < V; ++c) {
            ff.fx[c] = F3[c]; ff.fy[c] = F3[V + c]; ff.fz[c] = F3[2 * V + c];
        }
    }

public:
    QTensorSolver() = default;
    QTensorSolver(const QTensorSolver&) = delete;
    virtual ~QTensorSolver() { lbman_destroy(s_); }

    // Host initialisation with the reference's semantics
    // (src/qtensor_solver.tpp:14-48): director along z at the bulk order
    // S_eq (src/model.h:39-41), plus U(-NOISE, NOISE) on every component from
    // an unseeded generator.  Reproducible starts go through
    // lbman_init_seeded or lbman_upload instead.
    virtual void Initialize(QTensorFields& qf) const {
        const double s_eq = (-Params::B + std::sqrt(Params::B * Params::B - 24.0 * Params::A * Params::C)) /
                            (4.0 * Params::C);
        std::random_device rd;
        std::mt19937 gen(rd());
        std::uniform_real_distribution<double> noise(-Params::NOISE, Params::NOISE);
        const int64_t V = volume(qf.grid);
        for (int64_t c = 0; c < V; ++c) {
            qf.qxx[c] = -s_eq / 3.0 + noise(gen);
            qf.qxy[c] = noise(gen);
            qf.qxz[c] = noise(gen);
            qf.qyy[c] = -s_eq / 3.0 + noise(gen);
            qf.qyz[c] = noise(gen);
        }
    }

    // Phase 1 (src/qtensor_solver.tpp:51-147) on the GPU.
    void StepAndSetupBodyForce(QTensorFields& qf, FluidFields& ff) const {
        const int64_t V = volume(qf.grid);
        lbman_solver* s = get(qf.grid);
        lbman_dropin::Staging st;
        st.from_fields(ff, qf, V);
        lbman_dropin::check(lbman_upload(s, ff.rho.data(), st.u3.data(), st.q5.data(), nullptr, nullptr));
        lbman_dropin::check(lbman_qtensor_setup(s));
        std::vector<double> sig(5 * V), tau(3 * V);
        lbman_dropin::check(lbman_download(s, nullptr, nullptr, st.q5.data(), nullptr, st.F3.data()));
        lbman_dropin::check(lbman_download_stress(s, sig.data(), tau.data()));
        store_q(qf, st.q5, V);
        store_force(ff, st.F3, V);
        std::vector<double>* S[5] = {&qf.Sigma_xx, &qf.Sigma_xy, &qf.Sigma_xz, &qf.Sigma_yy, &qf.Sigma_yz};
        std::vector<double>* T[3] = {&qf.Tau_xy, &qf.Tau_xz, &qf.Tau_yz};
        for (int64_t c = 0; c < V; ++c) {
            for (int k = 0; k < 5; ++k) (*S[k])[c] = sig[k * V + c];
            for (int k = 0; k < 3; ++k) (*T[k])[c] = tau[k * V + c];
        }
    }

    // Phase 2, the base activity model (src/qtensor_solver.tpp:155-217), on
    // the GPU: ff.f* += -ALPHA div Q + div(Sigma + tau) - MU u.
    virtual void SetActiveStressAndComputeBodyForce(FluidFields& ff, const QTensorFields& qf) const {
        const int64_t V = volume(qf.grid);
        lbman_solver* s = get(qf.grid);
        lbman_dropin::Staging st;
        st.from_fields(ff, qf, V);
        std::vector<double> sig(5 * V), tau(3 * V);
        const std::vector<double>* S[5] = {&qf.Sigma_xx, &qf.Sigma_xy, &qf.Sigma_xz, &qf.Sigma_yy, &qf.Sigma_yz};
        const std::vector<double>* T[3] = {&qf.Tau_xy, &qf.Tau_xz, &qf.Tau_yz};
        for (int64_t c = 0; c < V; ++c) {
            for (int k = 0; k < 5; ++k) sig[k * V + c] = (*S[k])[c];
            for (int k = 0; k < 3; ++k) tau[k * V + c] = (*T[k])[c];
        }
        lbman_dropin::check(lbman_upload(s, ff.rho.data(), st.u3.data(), st.q5.data(), nullptr, st.F3.data()));
        lbman_dropin::check(lbman_upload_stress(s, sig.data(), tau.data()));
        lbman_dropin::check(lbman_active_force(s));
        lbman_dropin::check(lbman_download(s, nullptr, nullptr, nullptr, nullptr, st.F3.data()));
        store_force(ff, st.F3, V);
    }

    void Step(QTensorFields& qf, FluidFields& ff) const {
        if (typeid(*this) == typeid(QTensorSolver)) {
            StepFused(qf, ff);
            return;
        }
        StepAndSetupBodyForce(qf, ff);
        SetActiveStressAndComputeBodyForce(ff, qf);
    }

private:
    // Both phases of the base class in one GPU pass (lbman_qtensor_step).
    void StepFused(QTensorFields& qf, FluidFields& ff) const {
        const int64_t V = volume(qf.grid);
        lbman_solver* s = get(qf.grid);
        lbman_dropin::Staging st;
        st.from_fields(ff, qf, V);
        lbman_dropin::check(lbman_upload(s, ff.rho.data(), st.u3.data(), st.q5.data(), nullptr, nullptr));
        lbman_dropin::check(lbman_qtensor_step(s));
        lbman_dropin::check(lbman_download(s, nullptr, nullptr, st.q5.data(), nullptr, st.F3.data()));
        store_q(qf, st.q5, V);
        store_force(ff, st.F3, V);
    }
};

}  // namespace lbman
