"""The C++ drop-in (include/lbman3d_dropin.hpp) against the reference's own
solver classes, bit for bit, in FP64.

oracle/_ref/d_box/dropin_check (built by oracle/build_ref.py from the
reference sources beside the drop-in header, linked against
liblbman3d_b200.so) runs, for FullyPeriodic, Slit, Channel and a mixed
anchoring / moving-wall box of 10x12x8 cells:
  * ActiveNematicSim's GPU call sequence (src/active_nematic.h:51-108) through
    DeviceFields / DeviceSolver<BC>, against the CPU sequence
    QTensorSolver::Step + LbmSolver::LatticeBoltzmannStep;
  * lbman::LbmSolver<BC> (src/lbm_solver.h:12-21) on host fields, populations
    included;
  * lbman::QTensorSolver<BC>::Step (src/qtensor_solver.h:51), new Q and the
    full body force;
  * StepAndSetupBodyForce alone: new and previous Q, Sigma, tau and the
    Ericksen seed;
  * subclasses written once over either class: an empty
    SetActiveStressAndComputeBodyForce (pure relaxation,
    src/qtensor_solver.h:21), an override that calls the base and adds a
    space-varying active term (src/qtensor_solver.h:11-19), and one that
    overrides only Initialize -- an override replaces the activity model on
    the GPU as it does in the reference.
"""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "d_box", "dropin_check")


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(EXE), reason="oracle/_ref/d_box/dropin_check not built")
@pytest.mark.parametrize("steps", [1, 6])
def test_dropin_bitwise(steps):
    r = subprocess.run([EXE, str(steps)], capture_output=True, text=True, timeout=300)
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert r.returncode == 0, r.stdout + r.stderr
    checks = {(x["check"], x["bc"]) for x in lines}
    names = {"sim", "lbm_init", "lbm", "q", "q_setup", "q_zero", "q_varying", "q_init_only"}
    assert {c for c, _ in checks} == names, lines
    assert len(checks) == len(names) * 4, lines
    for x in lines:
        assert x["mismatches"] == 0, x
