"""Parity of the two-points-per-thread FP32 Q+force kernel (csrc/qpair.cuh,
organisation LBMAN_KERNELS_SPLIT_PAIR) through the C ABI.

* Against the FP64 CPU oracle (pinned bitwise to the reference): the same
  relative max-norm bounds as the one-point FP32 kernel -- 1e-6 after one
  step, 2e-5 after 20 -- on every wall type (x-walls whose rules apply to one
  half of a pair, y/z walls, anchoring, moving walls), partial tiles in x and
  y, upwind advection, each compiled pair tile and both z schedules.
* Against the one-point FP32 kernel on the same state: rounding only.
* FP16 population storage with the pair kernel.
"""
import numpy as np
import pytest

import lbman3d_b200 as L
from oracle import oracle as O

pytestmark = pytest.mark.gpu

PAIR = L._native.KERNELS_SPLIT_PAIR


def relerr(a, b):
    d = np.max(np.abs(np.asarray(a) - np.asarray(b)))
    s = np.max(np.abs(b))
    return d / s if s > 0 else d


def _case(grid, faces, upwind, seed=3, **phys):
    nx, ny, nz = grid
    p = O.make_params(nx, ny, nz, faces, O.UPWIND if upwind else O.CENTRED, **phys)
    V = nx * ny * nz
    q = O.seeded_q(p, seed, O.equilibrium_order(p), 1e-3)
    rng = np.random.default_rng(seed)
    rho = 1.0 + 0.01 * rng.standard_normal(V)
    u = 0.005 * rng.standard_normal(3 * V)
    return p, rho, u, q


def _sim(grid, faces, phys, upwind, precision=L.Precision.FP32, kernels=PAIR, tile=None):
    nx, ny, nz = grid
    p = L.Params(nx=nx, ny=ny, nz=nz, kQAdvection=L.Advection.Upwind if upwind else L.Advection.Centred, **phys)
    return L.Simulation(p, L.from_face_tuples(faces), precision, kernels, tile=tile)


# nx a multiple of 4 (16-byte staging); none is a multiple of 30, so every
# box has a partial tile in x
CASES = [
    ("periodic", (64, 20, 16), False),
    ("channel", (32, 26, 12), False),
    ("slit", (64, 33, 18), True),
    ("box_mixed", (36, 17, 19), False),
    ("lid", (44, 9, 14), True),
    ("qmixed", (20, 14, 13), True),
    ("walls", (40, 10, 9), False),
    ("anchored_z", (32, 12, 11), False),
]
TILES = [(30, 6, 0), (30, 10, 5), (30, 14, 0), (30, 10, 3)]


@pytest.mark.parametrize("tile", TILES, ids=[f"{t[0]}x{t[1]}z{t[2]}" for t in TILES])
@pytest.mark.parametrize("bc,grid,upwind", CASES, ids=[c[0] for c in CASES])
def test_pair_kernel_vs_fp64_oracle(bc, grid, upwind, tile):
    from cases import BC
    phys = dict(ALPHA=0.015, MU=0.002)
    p, rho, u, q = _case(grid, BC[bc], upwind, **phys)
    ref = O.OracleSim(p)
    ref.set(rho, u, q)
    sim = _sim(grid, BC[bc], phys, upwind, tile=tile)
    assert sim.shape()["kernels"] == PAIR
    sim.upload(rho, u, q)
    for n, tol in ((1, 1e-6), (19, 2e-5)):
        ref.step(n)
        sim.step(n)
        a, b = sim.download(), ref.get()
        for f in ("rho", "u", "q"):
            e = relerr(a[f], b[f])
            assert e <= tol, (bc, f, n, e)
    sim.close()


@pytest.mark.parametrize("bc,grid,upwind", CASES[:4], ids=[c[0] for c in CASES[:4]])
def test_pair_kernel_vs_one_point_kernel(bc, grid, upwind):
    from cases import BC
    phys = dict(ALPHA=0.01)
    _, rho, u, q = _case(grid, BC[bc], upwind, **phys)
    outs = []
    for kernels, tile in ((L._native.KERNELS_SPLIT, (32, 8, 0)), (PAIR, (30, 10, 0))):
        sim = _sim(grid, BC[bc], phys, upwind, kernels=kernels, tile=tile)
        sim.upload(rho, u, q)
        sim.qtensor_step()
        outs.append(sim.download(force=True))
        sim.close()
    for f in ("q", "force"):
        e = relerr(outs[1][f], outs[0][f])
        assert e <= 2e-6, (f, e)


@pytest.mark.parametrize("bc", ["periodic", "slit"])
def test_pair_kernel_fp16_storage_vs_fp64_oracle(bc):
    from cases import BC
    grid = {"periodic": (32, 18, 16), "slit": (32, 20, 14)}[bc]
    p, rho, u, q = _case(grid, BC[bc], False, ALPHA=0.01)
    ref = O.OracleSim(p)
    ref.set(rho, u, q)
    sim = _sim(grid, BC[bc], dict(ALPHA=0.01), False, precision=L.Precision.FP16, tile=(30, 10, 0))
    sim.upload(rho, u, q)
    for n, tol in ((1, 1e-3), (19, 1e-2)):
        ref.step(n)
        sim.step(n)
        a, b = sim.download(), ref.get()
        for f in ("rho", "u", "q"):
            assert relerr(a[f], b[f]) <= tol, (f, n)
    sim.close()


def test_pair_organisation_rejected_where_it_cannot_run():
    from cases import BC
    with pytest.raises(L._native.LbmanError):  # FP64 keeps the reference's arithmetic
        _sim((32, 8, 8), BC["periodic"], {}, False, precision=L.Precision.FP64, tile=(30, 10, 0))
    with pytest.raises(L._native.LbmanError):  # nx not a multiple of 4
        _sim((30, 8, 8), BC["periodic"], {}, False, tile=(30, 10, 0))
