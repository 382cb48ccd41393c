"""Long chaotic runs matched statistically (the reference's correctness check
for runs whose trajectories diverge): FP32 and FP16-storage runs against the
FP64 run -- bitwise the reference's arithmetic -- from the same seeded state,
compared on time-averaged defect density, mean |u|, the kinetic-energy
spectrum and the Q correlation length.
"""
import numpy as np
import pytest

import lbman3d_b200 as L

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

GRID = (48, 48, 48)
STEPS, WINDOW, EVERY = 1500, 500, 25


def _run(prec):
    nx, ny, nz = GRID
    p = L.Params(nx=nx, ny=ny, nz=nz, ALPHA=0.01)
    rows = []
    with L.Simulation(p, L.FullyPeriodicConfig(), prec) as sim:
        sim.init_seeded(4242, L.EquilibriumScalarOrder(p), 1e-3)
        sim.step(STEPS - WINDOW)
        for _ in range(WINDOW // EVERY):
            sim.step(EVERY)
            st = sim.statistics()
            E, _ = sim.velocity_spectrum(24)
            _, _, xi = sim.q_correlation(24)
            rows.append((st["defect_density"], st["mean_speed"], xi, E))
    dd = np.mean([r[0] for r in rows])
    ms = np.mean([r[1] for r in rows])
    xi = np.mean([r[2] for r in rows])
    E = np.mean([r[3] for r in rows], axis=0)
    return dd, ms, xi, E


@pytest.mark.parametrize("prec", [L.Precision.FP32, L.Precision.FP16], ids=["fp32", "fp16"])
def test_long_run_statistics_match_fp64(prec):
    ref = _run(L.Precision.FP64)
    got = _run(prec)
    assert ref[0] > 0 and ref[1] > 0
    for name, a, b in (("defect_density", got[0], ref[0]), ("mean_speed", got[1], ref[1]), ("xi", got[2], ref[2])):
        assert abs(a - b) <= 0.05 * abs(b), (name, a, b)
    E, Er = got[3][1:12], ref[3][1:12]
    assert np.linalg.norm(E - Er) <= 0.10 * np.linalg.norm(Er)
