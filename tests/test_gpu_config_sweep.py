"""The channel and slit workloads of the reference's stability envelope
(src/sim_config.h:30-34, 60-70): ChannelConfig (no-slip Neumann walls in x and
y, periodic z) at 20x100x100 and SlitConfig (free-slip walls confining x) at
64x256x256, params.h defaults, zeta (ALPHA) in {0.005, 0.01, 0.02}, centred
and upwind advection, 10^4 steps from the seeded random-director state, in
FP64 (bitwise the reference's arithmetic) and FP32.

Both runs must stay finite for the whole run (the envelope: LAMBDA = 0.3 is
inside the reliable range of both advection schemes, and free-slip
divergence sets in only after 1.1-1.6 * 10^4 steps), and since the active flow
is chaotic the FP32 run is matched to the FP64 one statistically over the
last 5000 steps, sampled every 50 (the correctness criterion for long
runs): mean |u| and
defect density within 5%, the kinetic-energy spectrum (shells 1-11) within
10% -- or, where the flow's own variability over that window is larger,
within twice the difference between the FP64 run and a second FP64 run whose
initial order parameter is perturbed by one part in 10^6 (the chaotic
spread of the statistic itself, measured on the reference arithmetic).
"""
import numpy as np
import pytest

import lbman3d_b200 as L

pytestmark = [pytest.mark.gpu, pytest.mark.slow]

STEPS, WINDOW, EVERY = 10000, 5000, 50
GEOM = {"channel": ((20, 100, 100), L.ChannelConfig), "slit": ((64, 256, 256), L.SlitConfig)}


def _run(geom, zeta, upwind, prec, perturb=0.0):
    (nx, ny, nz), bc = GEOM[geom]
    p = L.Params(nx=nx, ny=ny, nz=nz, ALPHA=zeta,
                 kQAdvection=L.Advection.Upwind if upwind else L.Advection.Centred)
    rows = []
    with L.Simulation(p, bc(), prec) as sim:
        sim.init_seeded(2718, L.EquilibriumScalarOrder(p) * (1.0 + perturb), 1e-3)
        sim.step(STEPS - WINDOW)
        for _ in range(WINDOW // EVERY):
            sim.step(EVERY)
            d = sim.reduce(L._native.DIAG_FLOW, raise_on_nan=False)
            assert not d["nan_detected"], (geom, zeta, upwind, prec)
            st = sim.statistics()
            E, _ = sim.velocity_spectrum(16)
            rows.append((st["defect_density"], st["mean_speed"], E))
    return (np.mean([r[0] for r in rows]), np.mean([r[1] for r in rows]), np.mean([r[2] for r in rows], axis=0))


@pytest.mark.parametrize("upwind", [False, True], ids=["centred", "upwind"])
@pytest.mark.parametrize("zeta", [0.005, 0.01, 0.02])
@pytest.mark.parametrize("geom", ["channel", "slit"])
def test_fp32_matches_fp64_over_ten_thousand_steps(geom, zeta, upwind):
    ref = _run(geom, zeta, upwind, L.Precision.FP64)
    got = _run(geom, zeta, upwind, L.Precision.FP32)
    assert ref[1] > 0
    checks = [("mean_speed", abs(got[1] - ref[1]), 0.05 * ref[1], 1),
              ("defect_density", abs(got[0] - ref[0]), 0.05 * max(ref[0], 1e-4), 0),
              ("spectrum", np.linalg.norm(got[2][1:12] - ref[2][1:12]), 0.10 * np.linalg.norm(ref[2][1:12]), 2)]
    if any(d > tol for _, d, tol, _ in checks):
        twin = _run(geom, zeta, upwind, L.Precision.FP64, perturb=1e-6)
        spread = [abs(twin[0] - ref[0]), abs(twin[1] - ref[1]), np.linalg.norm(twin[2][1:12] - ref[2][1:12])]
        for name, d, tol, k in checks:
            assert d <= max(tol, 2.0 * spread[k]), (name, d, tol, spread[k])
