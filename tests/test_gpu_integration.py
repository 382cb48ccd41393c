"""The reference's integration suite re-expressed on the GPU path
(tests/integration/*.cc): the same scenarios, parameters and assertions,
driven through the C ABI instead of the CPU solvers.
"""
import math

import numpy as np
import pytest

import lbman3d_b200 as L
from lbman3d_b200 import _native as N

pytestmark = pytest.mark.gpu


def mk(p, bc, precision=L.Precision.FP64):
    return L.Simulation(p, bc, precision)


def test_poiseuille_profile_symmetry_mass():
    """tests/integration/test_poiseuille.cc:112-135 (params tests/params/poiseuille)."""
    nx, ny, nz = 5, 16, 5
    TAUF = math.sqrt(float(np.float32(3.0) / np.float32(16.0))) + 0.5
    nu = (2 * TAUF - 1) / float(np.float32(6.0))
    u_max = 0.1
    dP = 8 * nu * u_max / float(ny * ny)
    p = L.Params(nx=nx, ny=ny, nz=nz, TAUF=TAUF, L=0.01, ALPHA=0.0)
    bc = L.BCConfig(L.WallSpec(L.Periodic(), L.Periodic()), L.WallSpec(L.Periodic(), L.Periodic()),
                    L.WallSpec(L.Neumann(), L.NoSlip()), L.WallSpec(L.Neumann(), L.NoSlip()),
                    L.WallSpec(L.Periodic(), L.Periodic()), L.WallSpec(L.Periodic(), L.Periodic()))
    V = nx * ny * nz
    force = np.zeros(3 * V)
    force[:V] = dP
    sim = mk(p, bc)
    sim.upload(np.ones(V), np.zeros(3 * V), np.zeros(5 * V), None, force)
    for _ in range(5000):
        sim.lbm_step()
    out = sim.download()
    ux = out["u"][:V].reshape(nz, ny, nx)
    prof = ux[nz // 2].mean(axis=1)
    y = np.arange(ny)
    analytic = dP / (2 * nu) * (y + 0.5) * (ny - 0.5 - y)
    assert np.max(np.abs(prof - analytic)) < 1e-4
    assert np.max(np.abs(prof[: ny // 2] - prof[::-1][: ny // 2])) < 1e-8
    tol = V * 5000 * np.finfo(float).eps
    assert abs(out["rho"].sum() - V) < tol


BC8 = dict(nx=8, ny=8, nz=16, TAUF=1.5, L=0.3, ALPHA=0.0)  # tests/params/bc_check


def test_fully_periodic_mass_conservation():
    """tests/integration/test_bc_combinations.cc:134-145"""
    p = L.Params(**BC8)
    V = p.V
    sim = mk(p, L.FullyPeriodicConfig())
    sim.upload(np.ones(V), np.zeros(3 * V), np.zeros(5 * V))
    m0 = sim.download()["rho"].sum()
    for _ in range(500):
        sim.lbm_step()
    m1 = sim.download()["rho"].sum()
    assert abs(m1 - m0) < V * 500 * np.finfo(float).eps


def test_channel_noslip_walls_damping():
    """tests/integration/test_bc_combinations.cc:152-173"""
    p = L.Params(**BC8)
    V = p.V
    u = np.zeros(3 * V)
    u[:V] = 0.01
    sim = mk(p, L.ChannelConfig())
    sim.upload(np.ones(V), u, np.zeros(5 * V))
    m0 = sim.download()["rho"].sum()
    for _ in range(500):
        sim.lbm_step()
    out = sim.download()
    assert abs(out["rho"].sum() - m0) < V * 500 * np.finfo(float).eps
    ux = out["u"][:V].reshape(p.nz, p.ny, p.nx)
    assert np.max(np.abs(ux[:, 0, :])) < 1e-6
    assert np.max(np.abs(ux[:, -1, :])) < 1e-6


def test_specular_z_free_slip():
    """tests/integration/test_bc_combinations.cc:182-212"""
    p = L.Params(**BC8)
    V = p.V
    bc = L.BCConfig(*([L.WallSpec(L.Periodic(), L.Periodic())] * 4),
                    L.WallSpec(L.Neumann(), L.SpecularReflection()), L.WallSpec(L.Neumann(), L.SpecularReflection()))
    force = np.zeros(3 * V)
    force[:V] = 1e-5
    sim = mk(p, bc)
    sim.upload(np.ones(V), np.zeros(3 * V), np.zeros(5 * V), None, force)
    for _ in range(500):
        sim.lbm_step()
    out = sim.download()
    ux = out["u"][:V].reshape(p.nz, p.ny, p.nx)
    uz = out["u"][2 * V:].reshape(p.nz, p.ny, p.nx)
    x0, y0 = p.nx // 2, p.ny // 2
    assert np.max(np.abs(ux[:, y0, x0] - ux[p.nz // 2, y0, x0])) < 1e-9
    assert np.max(np.abs(uz[0])) < 1e-9 and np.max(np.abs(uz[-1])) < 1e-9


def test_anchoring_converges_at_wall():
    """tests/integration/test_bc_combinations.cc:219-247 (Q only, u = 0)."""
    p = L.Params(**BC8)
    V = p.V
    anc = L.Anchoring(0.5, math.pi / 4.0, 0.0)
    bc = L.BCConfig(*([L.WallSpec(L.Periodic(), L.Periodic())] * 4), L.WallSpec(anc, L.NoSlip()),
                    L.WallSpec(anc, L.NoSlip()))
    rng = np.random.default_rng(42)
    q = np.concatenate([0.33 + rng.uniform(-0.05, 0.05, V), rng.uniform(-0.05, 0.05, V),
                        rng.uniform(-0.05, 0.05, V), -0.15 + rng.uniform(-0.05, 0.05, V),
                        rng.uniform(-0.05, 0.05, V)])
    sim = mk(p, bc)
    sim.upload(np.ones(V), np.zeros(3 * V), q)
    for _ in range(500):
        sim.qtensor_step()
    Q = sim.download()["q"].reshape(5, p.nz, p.ny, p.nx)
    target = L.boundary.anchored_q(anc)
    for k in range(5):
        assert np.max(np.abs(Q[k, 0] - target[k])) < 0.01


def _distorted_q(V, seed=42):
    rng = np.random.default_rng(seed)
    return np.concatenate([0.33 + rng.uniform(-0.05, 0.05, V), rng.uniform(-0.05, 0.05, V),
                           rng.uniform(-0.05, 0.05, V), -0.15 + rng.uniform(-0.05, 0.05, V),
                           rng.uniform(-0.05, 0.05, V)])


def test_coupled_backflow_relaxes():
    """tests/integration/test_coupled_backflow.cc:228-318 (16^3 passive, 2000 steps)."""
    p = L.Params(nx=16, ny=16, nz=16, TAUF=1.5, L=0.01, ALPHA=0.0)
    V = p.V
    sim = mk(p, L.FullyPeriodicConfig())
    sim.upload(np.ones(V), np.zeros(3 * V), _distorted_q(V))
    d0 = sim.reduce(N.DIAG_FLOW | N.DIAG_ENERGY)
    assert abs(d0["mass"] - V) < 1e-9
    ke, tot, mass = [d0["kinetic_energy"]], [d0["kinetic_energy"] + d0["free_energy"]], [d0["mass"]]
    max_speed = 0.0
    for i in range(200):
        sim.step(10)
        d = sim.reduce(N.DIAG_FLOW | N.DIAG_ENERGY)
        ke.append(d["kinetic_energy"])
        tot.append(d["kinetic_energy"] + d["free_energy"])
        mass.append(d["mass"])
        max_speed = max(max_speed, math.sqrt(d["umax2"]))
    assert ke[0] == 0.0
    assert max(ke) > 1e-16
    assert all(abs(m / mass[0] - 1.0) < 1e-10 for m in mass)
    assert all(k <= ke[1] * (1 + 1e-9) for k in ke[1:])
    assert ke[-1] / max(ke) < 1e-3
    assert all(t <= tot[0] + 1e-9 for t in tot[1:])
    assert tot[-1] < tot[0]
    assert max_speed < 0.1


def test_qtensor_relaxation_to_equilibrium_order():
    """tests/integration/test_qtensor_relaxation.cc:146-168 (16^3, u = 0, 2000 steps)."""
    p = L.Params(nx=16, ny=16, nz=16, TAUF=1.5, L=0.01, ALPHA=0.0)
    V = p.V
    sim = mk(p, L.FullyPeriodicConfig())
    sim.upload(np.ones(V), np.zeros(3 * V), _distorted_q(V))
    energies = []
    for i in range(2000):
        if i % 100 == 0:
            energies.append(sim.reduce(N.DIAG_ENERGY)["free_energy"])
        sim.qtensor_step()
    for a, b in zip(energies, energies[1:]):
        assert b < a + 1e-10
    assert energies[-2] - energies[-1] < 1e-6
    from oracle import oracle as O
    q = sim.download()["q"]
    op = O.make_params(16, 16, 16, [(0, (0, 0, 0), 0, (0, 0, 0))] * 6)
    S, _ = O.order_director(op, q)
    assert abs(S.mean() - (-p.B / (3.0 * p.C))) < 1e-6
    assert S.std() < 1e-2
