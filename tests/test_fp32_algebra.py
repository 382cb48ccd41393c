"""The FP32 arithmetic rearrangements.  The Q-stage right-hand side (csrc/physics.cuh pointwise_q_mat) is an
algebraic rearrangement of the reference's term-by-term expansion
(pointwise_q, src/model.h:102-342).  Compiled here as host C++ in double
precision, the two must agree to rounding on random states."""
import os
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(os.path.dirname(HERE), "lbman3d_b200", "csrc")


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_fp32_rhs_matches_reference_form(tmp_path):
    exe = str(tmp_path / "algebra_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(HERE, "host", "stub"), "-I", CSRC,
                    os.path.join(HERE, "host", "algebra_check.cpp"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_fp32_paired_relaxation_matches_reference_form(tmp_path):
    """The FP32 BGK + Guo relaxation by opposite direction pairs
    (csrc/lbm.cuh relax_pairs) against the direction-by-direction form of the
    reference (src/physics_helpers.h:69-129), in double, with and without
    deviation storage."""
    exe = str(tmp_path / "collide_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(HERE, "host", "stub"), "-I", CSRC,
                    os.path.join(HERE, "host", "collide_check.cpp"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_packed_pair_rhs_matches_reference_form(tmp_path):
    """The two-point packed FP32 right-hand side (csrc/physics_pair.cuh
    pointwise_q_pair: Q_new, row stress, Ericksen force) against the
    reference-ordered pointwise_q in double, per point, centred and upwind;
    FP32 rounding only."""
    exe = str(tmp_path / "pair_check")
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(HERE, "host", "stub"), "-I", CSRC,
                    os.path.join(HERE, "host", "pair_check.cpp"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 0, r.stdout + r.stderr
