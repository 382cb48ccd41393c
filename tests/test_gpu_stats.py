"""Flow / order statistics on the GPU against the NumPy oracle
(oracle/stats.py): kinetic-energy spectrum, Q autocorrelation and
correlation length, mean / rms speed, defect density.  Parity for these rows
is unpinned by the reference (it has no such analysis); the oracle is pinned
to direct sums and Parseval in tests/test_oracle_stats.py.
"""
import math

import numpy as np
import pytest

import lbman3d_b200 as L
from oracle import stats as S

pytestmark = pytest.mark.gpu

CASES = [((16, 16, 16), "periodic"), ((12, 20, 9), "slit"), ((7, 10, 13), "channel")]
BC = {"periodic": L.FullyPeriodicConfig, "slit": L.SlitConfig, "channel": L.ChannelConfig}
TOL = {L.Precision.FP64: 1e-10, L.Precision.FP32: 2e-5}


def _fields(grid, seed):
    nx, ny, nz = grid
    V = nx * ny * nz
    r = np.random.default_rng(seed)
    rho = 1.0 + 0.01 * r.standard_normal(V)
    u = 0.02 * r.standard_normal((3, V))
    q = 0.1 * r.standard_normal((5, V))
    return rho, u, q


def _sim(grid, bc, prec):
    nx, ny, nz = grid
    return L.Simulation(L.Params(nx=nx, ny=ny, nz=nz), BC[bc](), prec)


@pytest.mark.parametrize("prec", [L.Precision.FP64, L.Precision.FP32], ids=["fp64", "fp32"])
@pytest.mark.parametrize("grid,bc", CASES)
def test_spectrum_matches_oracle(grid, bc, prec):
    rho, u, q = _fields(grid, 11)
    with _sim(grid, bc, prec) as sim:
        sim.upload(rho, u.ravel(), q.ravel())
        nb = sim.default_bins()
        E, cnt = sim.velocity_spectrum(nb)
        got_u = sim.download()["u"]
    Eo, co = S.velocity_spectrum(got_u, *grid, nb)
    np.testing.assert_array_equal(cnt, co)
    assert np.max(np.abs(E - Eo)) <= TOL[prec] * np.max(Eo)
    # Parseval: every shell is covered
    assert math.isclose(E.sum(), 0.5 * np.mean(np.sum(got_u.reshape(3, -1) ** 2, axis=0)), rel_tol=10 * TOL[prec])


@pytest.mark.parametrize("prec", [L.Precision.FP64, L.Precision.FP32], ids=["fp64", "fp32"])
@pytest.mark.parametrize("grid,bc", CASES)
def test_q_correlation_matches_oracle(grid, bc, prec):
    rho, u, q = _fields(grid, 12)
    # a smooth, correlated Q: low-pass the noise along every axis
    nx, ny, nz = grid
    g = q.reshape(5, nz, ny, nx)
    for ax in (1, 2, 3):
        g = (g + np.roll(g, 1, axis=ax) + np.roll(g, -1, axis=ax)) / 3.0
    q = g.reshape(5, -1)
    with _sim(grid, bc, prec) as sim:
        sim.upload(rho, u.ravel(), q.ravel())
        nb = sim.default_bins()
        C, cnt, xi = sim.q_correlation(nb)
        got_q = sim.download()["q"]
    Co, co, xio = S.q_correlation(got_q, *grid, nb)
    np.testing.assert_array_equal(cnt, co)
    assert np.max(np.abs(C - Co)) <= 10 * TOL[prec]
    assert C[0] == pytest.approx(1.0, abs=1e-12)
    assert xio > 0 and abs(xi - xio) <= 1e3 * TOL[prec]


def test_single_mode_spectrum():
    nx, ny, nz = 16, 24, 8
    V = nx * ny * nz
    A, m = 0.05, 3
    y = np.arange(ny)
    ux = np.broadcast_to(A * np.sin(2 * np.pi * m * y / ny)[None, :, None], (nz, ny, nx)).ravel()
    u = np.concatenate([ux, np.zeros(2 * V)])
    with _sim((nx, ny, nz), "periodic", L.Precision.FP64) as sim:
        sim.upload(np.ones(V), u, np.zeros(5 * V))
        E, _ = sim.velocity_spectrum()
    b = int(math.floor(max(nx, ny, nz) * m / ny + 0.5))
    assert E[b] == pytest.approx(A * A / 4, rel=1e-12)
    assert abs(E.sum() - E[b]) < 1e-15


@pytest.mark.parametrize("prec", [L.Precision.FP64, L.Precision.FP32], ids=["fp64", "fp32"])
def test_statistics_scalars(prec):
    grid = (12, 14, 10)
    rho, u, q = _fields(grid, 13)
    with _sim(grid, "periodic", prec) as sim:
        sim.upload(rho, u.ravel(), q.ravel())
        st = sim.statistics()
        d = sim.reduce(L._native.DIAG_DEFECTS)
        got_u = sim.download()["u"]
    m1, m2 = S.speed_moments(got_u, int(np.prod(grid)))
    assert st["mean_speed"] == pytest.approx(m1, rel=1e-12)
    assert st["rms_speed"] == pytest.approx(math.sqrt(m2), rel=1e-12)
    assert st["defect_faces"] == d["defect_faces"] and st["defect_faces"] > 0
    assert st["defect_density"] == pytest.approx(d["defect_faces"] / np.prod(grid))


def test_statistics_after_steps_and_bad_bins():
    grid = (16, 16, 16)
    with _sim(grid, "periodic", L.Precision.FP32) as sim:
        sim.init_seeded(5, 0.5, 1e-3)
        sim.step(20)
        E, _ = sim.velocity_spectrum()
        out = sim.download()
        assert E.sum() == pytest.approx(0.5 * np.mean(np.sum(out["u"].reshape(3, -1) ** 2, axis=0)), rel=1e-4)
        with pytest.raises(L._native.LbmanError):
            sim.velocity_spectrum(L._native.STATS_MAX_BINS + 1)
