"""Boundary configurations and golden cases shared by the fixture generator
(tests/golden/make_golden.py) and the parity tests.

Each face is (qbc, (S, theta, phi), ubc, (Ux, Uy, Uz)) in XLo, XHi, YLo,
YHi, ZLo, ZHi order, with qbc in {0 periodic, 1 neumann, 2 anchoring} and
ubc in {0 periodic, 1 noslip, 2 moving wall, 3 specular}.  The named
configurations mirror the ones oracle/ref_driver.cc instantiates from the
reference's type-level presets.
"""
import math

Z3 = (0.0, 0.0, 0.0)
PER = (0, Z3, 0, Z3)
NEU_NOSLIP = (1, Z3, 1, Z3)
NEU_SPEC = (1, Z3, 3, Z3)


def anch(S, th, ph, ubc=1, uw=Z3):
    return (2, (S, th, ph), ubc, uw)


BC = {
    "periodic": [PER] * 6,
    "channel": [NEU_NOSLIP] * 4 + [PER] * 2,
    "slit": [NEU_SPEC] * 2 + [PER] * 4,
    "slit_noslip": [NEU_NOSLIP] * 2 + [PER] * 4,
    "poiseuille": [PER, PER, NEU_NOSLIP, NEU_NOSLIP, PER, PER],
    "specular_z": [PER] * 4 + [NEU_SPEC] * 2,
    "anchored_z": [PER] * 4 + [anch(0.5, math.pi / 4.0, 0.0)] * 2,
    "lid": [PER, PER, NEU_NOSLIP, anch(0.4, 1.0, 0.3, 2, (0.05, 0.0, 0.02)), PER, PER],
    "box_mixed": [NEU_SPEC, anch(0.5, 0.7, 1.1, 3), NEU_NOSLIP, (1, Z3, 2, (0.03, 0.0, -0.01)),
                  anch(0.3, 0.2, 0.5, 1), (1, Z3, 2, (0.0, 0.02, 0.0))],
    "qmixed": [PER, (1, Z3, 0, Z3), anch(0.5, 0.3, 0.2, 0), anch(0.5, 0.3, 0.2, 0), NEU_SPEC, NEU_NOSLIP],
    "walls": [NEU_NOSLIP] * 6,
    # periodic Q with no-slip velocity walls on x (oracle-only larger-box case)
    "qper_uwall": [(0, Z3, 1, Z3)] * 2 + [PER] * 4,
}

# Compile-time parameter sets of oracle/build_ref.py (physics only).
PHYS = {
    "g_p8": dict(),
    "g_678": dict(ALPHA=0.02, MU=0.01),
    "g_678_up": dict(ALPHA=0.02),
    "g_thin": dict(),
    "g_unit": dict(DT=0.05, TAUF=1.5 * 0.05, L=0.01, ALPHA=0.04),
    "g_lbm": dict(TAUF=0.9330127018922193, ALPHA=0.0),
}
GRID = {"g_p8": (8, 8, 8), "g_678": (6, 7, 8), "g_678_up": (6, 7, 8), "g_thin": (1, 5, 6),
        "g_unit": (5, 5, 5), "g_lbm": (5, 16, 5)}
UPWIND = {"g_678_up"}

# name: (build, bc, mode, init, snapshots)
#   init: "baseline" = rho 1, u 0, seeded random director Q (S0 = S_eq, sigma 1e-3)
#         "perturbed" = baseline Q plus 1% density and 0.01 velocity noise
#         "force:<fx>" = rho 1, u 0, Q baseline, constant body force fx
CASES = {
    "periodic_p8": ("g_p8", "periodic", "full", "baseline", (1, 10)),
    "channel_678": ("g_678", "channel", "full", "perturbed", (1, 10)),
    "slit_678_upwind": ("g_678_up", "slit", "full", "perturbed", (1, 10)),
    "box_mixed_678": ("g_678", "box_mixed", "full", "perturbed", (1, 10)),
    "lid_678": ("g_678", "lid", "full", "perturbed", (1, 10)),
    "qmixed_678": ("g_678", "qmixed", "full", "perturbed", (1, 10)),
    "walls_678": ("g_678", "walls", "full", "perturbed", (1, 10)),
    "anchored_z_678_q": ("g_678", "anchored_z", "q", "perturbed", (1, 10)),
    "thin_box_mixed": ("g_thin", "box_mixed", "full", "perturbed", (1, 10)),
    "unit_periodic": ("g_unit", "periodic", "full", "perturbed", (1, 10)),
    "poiseuille_lbm": ("g_lbm", "poiseuille", "lbm", "force:3.125e-05", (1, 50)),
    "specular_z_lbm": ("g_p8", "specular_z", "lbm", "force:1e-05", (1, 20)),
}
