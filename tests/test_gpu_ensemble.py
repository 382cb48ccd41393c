"""Ensemble runner: every box of a batched run must match the same box run
alone through the single-box path bit for bit (the kernels do the same
arithmetic), through the CUDA-graph replay, in both kernel organisations and
in FP64 and FP32; the autotuner must leave every box's state untouched."""
import numpy as np
import pytest

import lbman3d_b200 as L
from lbman3d_b200 import _native as N

pytestmark = pytest.mark.gpu


def _boxes():
    from cases import BC
    specs = [((20, 18, 16), "periodic", dict(ALPHA=0.01, LAMBDA=0.2)),
             ((24, 12, 30), "slit", dict(ALPHA=0.02, LAMBDA=0.5)),
             ((9, 13, 11), "box_mixed", dict(ALPHA=0.005, MU=0.01)),
             ((33, 7, 10), "channel", dict(ALPHA=0.015)),
             ((16, 16, 16), "lid", dict(ALPHA=0.003, LAMBDA=0.65))]
    return [(L.Params(nx=g[0], ny=g[1], nz=g[2], **ph), L.from_face_tuples(BC[bc])) for g, bc, ph in specs]


def _inputs(p, seed):
    from oracle import oracle as O
    op = O.make_params(p.nx, p.ny, p.nz, [(0, (0, 0, 0), 0, (0, 0, 0))] * 6)
    q = O.seeded_q(op, seed, 0.5, 1e-3)
    rng = np.random.default_rng(seed)
    return 1.0 + 0.01 * rng.standard_normal(p.V), 0.004 * rng.standard_normal(3 * p.V), q


@pytest.mark.parametrize("precision", [L.Precision.FP64, L.Precision.FP32], ids=["fp64", "fp32"])
@pytest.mark.parametrize("kernels", [N.KERNELS_SPLIT, N.KERNELS_FUSED], ids=["split", "fused"])
def test_ensemble_boxes_match_single_box_runs_bitwise(precision, kernels):
    boxes = _boxes()
    ens = L.Ensemble(boxes, precision, kernels, tile=(14, 14, 0))
    singles = []
    for b, (p, bc) in enumerate(boxes):
        rho, u, q = _inputs(p, 100 + b)
        ens.upload(b, rho, u, q)
        s = L.Simulation(p, bc, precision)
        s.upload(rho, u, q)
        singles.append(s)
    nsteps = 27  # first step eager, 20 from a graph replay, 6 eager
    ens.step(nsteps)
    for s in singles:
        s.step(nsteps)
    info = ens.info()
    assert info["steps"] == nsteps and info["cells"] == sum(p.V for p, _ in boxes)
    for b, s in enumerate(singles):
        x, y = ens.download(b, f=True), s.download(f=True)
        for k in ("rho", "u", "q", "f"):
            np.testing.assert_array_equal(x[k], y[k], err_msg=f"box {b} field {k}")


def test_ensemble_autotune_restores_state_and_seeded_boxes_are_distinct():
    boxes = L.draw_boxes(6, seed=3)
    ens = L.Ensemble(boxes, L.Precision.FP32)
    ens.init_seeded(42)
    ens.step(3)
    before = [ens.download(b) for b in range(len(boxes))]
    best = ens.autotune(steps_per_trial=2)
    assert best["trials"] >= 6 and best["ms_per_step"] > 0
    after = [ens.download(b) for b in range(len(boxes))]
    for x, y in zip(before, after):
        for k in x:
            np.testing.assert_array_equal(x[k], y[k])
    assert not np.array_equal(before[0]["q"][:100], before[2]["q"][:100])
    ens.step(5)
    assert ens.info()["steps"] == 8


def test_draw_boxes_matches_the_batching_workload():
    boxes = L.draw_boxes(96, seed=0)
    assert len(boxes) == 96
    for i, (p, bc) in enumerate(boxes):
        for side in (p.nx, p.ny, p.nz):
            assert side in L.ensemble.SIDES
        assert p.ny == p.nz and p.nx <= p.ny
        assert 1e-3 <= p.ALPHA <= 3e-2 and 0.1 <= p.LAMBDA <= 0.7
        assert isinstance(bc, L.FullyPeriodicConfig if i % 2 == 0 else L.SlitConfig)


@pytest.mark.parametrize("world", [2, 3])
def test_sharded_ensemble_equals_the_whole_ensemble(world):
    """The ensemble split over ranks (emulated here as shards in one process
    on one GPU): every box, seeded by its index in the whole ensemble, ends
    bitwise where the unsharded ensemble leaves it."""
    boxes = _boxes()
    whole = L.Ensemble(boxes, L.Precision.FP32, N.KERNELS_SPLIT, tile=(14, 14, 0))
    whole.init_seeded(11)
    whole.step(6)
    for r in range(world):
        sh = L.ShardedEnsemble(boxes, r, world, L.Precision.FP32, N.KERNELS_SPLIT, tile=(14, 14, 0))
        sh.init_seeded(11)
        sh.step(6)
        for g in sh.ids:
            a, b = sh.download_box(g, f=True), whole.download(g, f=True)
            for k in ("rho", "u", "q", "f"):
                np.testing.assert_array_equal(a[k], b[k], err_msg=f"box {g} {k}")
        sh.close()
    whole.close()


def test_fp16_boxes_match_single_box_runs_bitwise():
    """FP16 population storage: a single box streams in place (AA pattern,
    one population buffer), the ensemble through its two-buffer kernel.  All
    forms do the same per-cell arithmetic and the same conversions, so every
    box matches bit for bit, after odd and even step counts."""
    from cases import BC
    # periodic boxes with even nx take the two-cells-per-thread kernels, odd
    # nx and walled boxes the one-cell kernels
    specs = [((24, 10, 12), "periodic"), ((40, 8, 6), "periodic"), ((8, 12, 10), "periodic"),
             ((21, 10, 8), "periodic"), ((24, 12, 30), "slit")]
    boxes = [(L.Params(nx=g[0], ny=g[1], nz=g[2], ALPHA=0.01), L.from_face_tuples(BC[bc])) for g, bc in specs]
    ens = L.Ensemble(boxes, L.Precision.FP16, N.KERNELS_SPLIT, tile=(14, 14, 0))
    singles = []
    for b, (p, bc) in enumerate(boxes):
        rho, u, q = _inputs(p, 200 + b)
        ens.upload(b, rho, u, q)
        s = L.Simulation(p, bc, L.Precision.FP16)
        s.upload(rho, u, q)
        singles.append(s)
    for n in (5, 2):
        ens.step(n)
        for s in singles:
            s.step(n)
        for b, s in enumerate(singles):
            x, y = ens.download(b, f=True), s.download(f=True)
            for k in ("rho", "u", "q", "f"):
                np.testing.assert_array_equal(x[k], y[k], err_msg=f"box {b} field {k} after {n}")
    for s in singles:
        s.close()
