"""The simulation driver (lbman3d_b200/sim.py): lbm.log number formatting
against C++ std::format, and (GPU) the main loop's log, frames and
divergence exit.

The format vectors were printed by g++ 13's std::format("{}", x) (C++20),
the formatter the reference's compat::println uses.
"""
import json
import math
import os

import numpy as np
import pytest

from lbman3d_b200.sim import cxx_format

VECTORS = [
    (0.0, "0"), (-0.0, "-0"), (1.0, "1"), (-1.0, "-1"), (0.5, "0.5"), (1e-05, "1e-05"), (100000.0, "1e+05"),
    (123456.0, "123456"), (0.0001, "1e-04"), (0.001, "0.001"), (1e16, "1e+16"), (1.5e-7, "1.5e-07"),
    (3.141592653589793, "3.141592653589793"), (2.5, "2.5"), (0.3333333333333333, "0.3333333333333333"),
    (262144.0, "262144"), (262144.00000000003, "262144.00000000006"), (1e-300, "1e-300"),
    (6.02214076e23, "6.02214076e+23"), (0.1, "0.1"), (12.0, "12"), (1234567.0, "1234567"), (1e21, "1e+21"),
    (0.00012345, "0.00012345"), (5e-324, "5e-324"), (1.7976931348623157e308, "1.7976931348623157e+308"),
    (7e-3, "0.007"), (0.07, "0.07"), (999999.0, "999999"), (1e6, "1e+06"), (65536.5, "65536.5"),
    (-2.5e-10, "-2.5e-10"), (math.nan, "nan"), (math.inf, "inf"),
]


@pytest.mark.parametrize("x,s", VECTORS)
def test_format_matches_std_format(x, s):
    assert cxx_format(x) == s


def test_format_integers_and_negative_nan():
    assert cxx_format(42) == "42" and cxx_format(np.int64(-7)) == "-7"
    assert cxx_format(math.copysign(math.nan, -1.0)) == "-nan"


@pytest.mark.gpu
def test_main_loop_log_frames_and_divergence(tmp_path):
    from lbman3d_b200 import sim as S
    log = tmp_path / "lbm.log"
    rc = S.main(["--nx", "12", "--ny", "10", "--nz", "8", "--bc", "channel", "--steps", "30",
                 "--save-interval", "10", "--export", str(tmp_path / "data"), "--log", str(log)])
    assert rc == 0
    text = log.read_text().splitlines()
    assert text[0].startswith("Hybrid Lattice Boltzmann simulation for 3D active nematics")
    assert "  nx = 12, ny = 10, nz = 8" in text and "  DX = 1, DY = 1, DZ = 1" in text
    rows = [t for t in text if t.startswith("Time ")]
    assert [r.split(":")[0] for r in rows] == ["Time 0", "Time 10", "Time 20"]
    for r in rows:
        fields = dict(kv.split(": ") for kv in r.split(": ", 1)[1].split(", "))
        assert abs(float(fields["Mass"]) - 960.0) < 1e-6
        assert int(fields["NumDisclinations"]) >= 0
        assert math.isfinite(float(fields["Max |u|"]))
    assert rows[0].split("Relative Error: ")[1].startswith("-nan")
    assert text[-1] == "LBM program exited."
    hdr = json.loads((tmp_path / "data" / "frame_000002.json").read_text())
    assert hdr["step"] == 20 and hdr["grid"] == [12, 10, 8]
    raw = (tmp_path / "data" / "frame_000002.bin").read_bytes()
    a = {e["name"]: e for e in hdr["arrays"]}
    rho = np.frombuffer(raw, dtype=a["rho"]["dtype"], count=960, offset=a["rho"]["offset"])
    assert abs(rho.sum() - 960.0) < 1e-6

    # divergence: a NaN density makes Log return False and write the notice
    d = S.ActiveNematicSim(S.Params(nx=6, ny=6, nz=6), S.BCS["periodic"](), log_path=str(tmp_path / "d.log"))
    V = 216
    rho = np.ones(V)
    rho[3] = np.nan
    d.sim.upload(rho, np.zeros(3 * V), np.zeros(5 * V))
    assert d.Log() is False
    d.close()
    assert any(t.startswith("DIVERGED at time step 0") for t in (tmp_path / "d.log").read_text().splitlines())
