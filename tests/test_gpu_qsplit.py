"""The Q stage as the reference's two phases (lbman_qtensor_setup =
QTensorSolver::StepAndSetupBodyForce, lbman_active_force = the base
SetActiveStressAndComputeBodyForce, src/qtensor_solver.tpp:51-217), and the
host-field QTensorSolver whose overrides replace the second phase.

* Against the golden fixtures of the reference's own CPU solver: FP64 bitwise,
  new Q, Sigma, tau and the body force, for every case (Q-only cases are the
  reference tests' zero-activity subclass: phase 1 alone).
* The two phases against the one-pass kernel: the same Q and force (bitwise
  in FP64, to rounding in FP32).
* The Python QTensorSolver: the base class (one fused pass), an empty
  override (pure relaxation) and an override that calls the base, against the
  CPU oracle's step with and without the activity phase.
"""
import numpy as np
import pytest

import lbman3d_b200 as L
from golden_util import load, names
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _sim(g, precision=L.Precision.FP64):
    nx, ny, nz = g["grid"]
    p = L.Params(nx=nx, ny=ny, nz=nz, kQAdvection=L.Advection.Upwind if g["upwind"] else L.Advection.Centred,
                 **g["phys"])
    return p, L.Simulation(p, L.from_face_tuples(g["faces"]), precision, L._native.KERNELS_SPLIT)


@pytest.mark.parametrize("name", names())
def test_two_phase_q_stage_matches_reference_bitwise(name):
    g = load(name)
    _, sim = _sim(g)
    sim.upload(g["in_rho"], g["in_u"], g["in_q"], None, g["in_force"])
    done = 0
    for k, t in enumerate(g["steps"]):
        for _ in range(t - done):
            if g["mode"] == "full":
                sim.qtensor_setup()
                sim.active_force()
                sim.lbm_step()
            elif g["mode"] == "q":
                sim.qtensor_setup()
            else:
                sim.lbm_step()
        done = t
        out = sim.download(f=True, force=True)
        fields = {"full": ("rho", "u", "q", "f", "force"), "q": ("q", "force"), "lbm": ("rho", "u", "f")}[g["mode"]]
        for f in fields:
            np.testing.assert_array_equal(out[f], g[f"s{k}_{f}"], err_msg=f"{name} step {t} {f}")
        if g["mode"] != "lbm":
            sig, tau = sim.download_stress()
            np.testing.assert_array_equal(sig, g[f"s{k}_sigma"], err_msg=f"{name} step {t} sigma")
            np.testing.assert_array_equal(tau, g[f"s{k}_tau"], err_msg=f"{name} step {t} tau")
    sim.close()


@pytest.mark.parametrize("name", ["periodic_p8", "walls_678", "box_mixed_678", "slit_678_upwind"])
@pytest.mark.parametrize("precision", [L.Precision.FP64, L.Precision.FP32], ids=["fp64", "fp32"])
def test_two_phases_equal_the_one_pass_kernel(name, precision):
    g = load(name)
    outs = []
    for two_phase in (False, True):
        _, sim = _sim(g, precision)
        sim.upload(g["in_rho"], g["in_u"], g["in_q"], None, g["in_force"])
        for _ in range(3):
            if two_phase:
                sim.qtensor_setup()
                sim.active_force()
            else:
                sim.qtensor_step()
            sim.lbm_step()
        outs.append(sim.download(force=True))
        sim.close()
    for f in ("rho", "u", "q", "force"):
        if precision == L.Precision.FP64:
            np.testing.assert_array_equal(outs[1][f], outs[0][f], err_msg=f)
        else:  # the one-pass FP32 kernel rearranges the right-hand side: rounding only
            d = np.max(np.abs(outs[1][f] - outs[0][f])) / max(np.max(np.abs(outs[0][f])), 1e-30)
            assert d <= 1e-4, (f, d)


class ZeroActivity(L.QTensorSolver):
    """Pure relaxation: the reference's empty override (src/qtensor_solver.h:21)."""

    def SetActiveStressAndComputeBodyForce(self, ff, qf):
        pass


class BasePlusExtra(L.QTensorSolver):
    """An override that calls the base activity model and adds a term."""

    def SetActiveStressAndComputeBodyForce(self, ff, qf):
        super().SetActiveStressAndComputeBodyForce(ff, qf)
        ff.fx += 1e-3


@pytest.mark.parametrize("name", ["box_mixed_678", "lid_678", "periodic_p8"])
@pytest.mark.parametrize("cls", [L.QTensorSolver, ZeroActivity, BasePlusExtra],
                         ids=["base", "zero", "base_plus_extra"])
def test_host_solver_override_replaces_the_activity_phase(name, cls):
    g = load(name)
    p, sim = _sim(g)
    sim.close()
    grid = L.LocalGrid.SingleRank(p)
    ff, qf = L.FluidFields(grid), L.QTensorFields(grid)
    V = p.V
    ff.rho[:] = g["in_rho"]
    ff.ux[:], ff.uy[:], ff.uz[:] = g["in_u"][:V], g["in_u"][V:2 * V], g["in_u"][2 * V:]
    qf.set_q5(g["in_q"])
    q_old = qf.q5().copy()
    solver = cls(L.from_face_tuples(g["faces"]), p)
    solver.Step(qf, ff)
    nx, ny, nz = g["grid"]
    op = O.make_params(nx, ny, nz, g["faces"], O.UPWIND if g["upwind"] else O.CENTRED, **g["phys"])
    ref = O.OracleSim(op)
    ref.set(g["in_rho"], g["in_u"], g["in_q"])
    ref.q_step(with_active=cls is not ZeroActivity)
    r = ref.get()
    np.testing.assert_array_equal(qf.q5(), r["q"])
    np.testing.assert_array_equal(np.concatenate([qf.qxx_new, qf.qxy_new, qf.qxz_new, qf.qyy_new, qf.qyz_new]),
                                  q_old)
    extra = 1e-3 if cls is BasePlusExtra else 0.0
    np.testing.assert_array_equal(ff.fx, r["force"][:V] + extra)
    np.testing.assert_array_equal(ff.fy, r["force"][V:2 * V])
    np.testing.assert_array_equal(ff.fz, r["force"][2 * V:])
    if cls is not L.QTensorSolver:  # the two-phase path fills the stresses
        sig = np.concatenate([getattr(qf, c) for c in L.QTensorSolver.SIGMA])
        tau = np.concatenate([getattr(qf, c) for c in L.QTensorSolver.TAU])
        np.testing.assert_array_equal(sig, r["sigma"])
        np.testing.assert_array_equal(tau, r["tau"])
    solver.sim.close()
