"""Autotuner: it must leave the state exactly as it found it, pick a compiled
shape, and -- since every kernel organisation and tile performs the same
arithmetic -- the tuned solver must stay bitwise equal to the untuned one."""
import numpy as np
import pytest

import lbman3d_b200 as L
from lbman3d_b200 import _native as N

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bc,grid", [("slit", (40, 36, 30)), ("periodic", (33, 20, 17))])
def test_autotune_restores_state_and_keeps_results(bc, grid):
    from cases import BC
    from oracle import oracle as O

    nx, ny, nz = grid
    p = L.Params(nx=nx, ny=ny, nz=nz, ALPHA=0.01)
    op = O.make_params(nx, ny, nz, BC[bc])
    q = O.seeded_q(op, 9, 0.5, 1e-3)
    V = p.V
    rng = np.random.default_rng(1)
    rho, u = 1.0 + 0.01 * rng.standard_normal(V), 0.005 * rng.standard_normal(3 * V)
    a = L.Simulation(p, L.from_face_tuples(BC[bc]), L.Precision.FP64)
    b = L.Simulation(p, L.from_face_tuples(BC[bc]), L.Precision.FP64)
    for s in (a, b):
        s.upload(rho, u, q)
        s.step(2)
    before = a.download(f=True, force=True)
    best = a.autotune(steps_per_trial=2)
    assert best["trials"] >= 6 and best["ms_per_step"] > 0
    assert best["kernels"] in (N.KERNELS_SPLIT, N.KERNELS_FUSED)
    assert a.shape()["tile_x"] == best["tile_x"]
    after = a.download(f=True, force=True)
    for k in before:
        np.testing.assert_array_equal(before[k], after[k], err_msg=k)
    assert a.steps_done() == 2
    a.step(5)
    b.step(5)
    x, y = a.download(f=True), b.download(f=True)
    for k in x:
        np.testing.assert_array_equal(x[k], y[k], err_msg=k)


def test_set_shape_rejects_uncompiled_tiles():
    p = L.Params(nx=16, ny=16, nz=16)
    s = L.Simulation(p, L.FullyPeriodicConfig(), L.Precision.FP64)
    with pytest.raises(N.LbmanError):
        s.set_shape(N.KERNELS_SPLIT, 62, 6, 8)  # does not fit FP64 shared memory
    with pytest.raises(N.LbmanError):
        s.set_shape(N.KERNELS_SPLIT, 17, 5, 8)
    s.set_shape(N.KERNELS_FUSED, 14, 14, 4)
    assert s.shape()["kernels"] == N.KERNELS_FUSED and s.shape()["threads"] == 256


def test_untuned_defaults():
    """The shape a handle starts with before any autotuning: the pair Q
    kernel under LBMAN_KERNELS_AUTO where its 30-wide tiles pad x by at most
    10% (FP32/FP16, nx a multiple of 4), else the one-point split kernel in
    32 x 8 tiles where those fit; fixed z chunks."""
    def shape(nx, ny, nz, prec):
        with L.Simulation(L.Params(nx=nx, ny=ny, nz=nz), L.FullyPeriodicConfig(), prec) as s:
            return s.shape()
    a = shape(120, 40, 40, L.Precision.FP32)  # 4 pair tiles exactly
    assert (a["kernels"], a["tile_x"], a["tile_y"]) == (N.KERNELS_SPLIT_PAIR, 30, 10)
    b = shape(64, 40, 40, L.Precision.FP32)  # 30-wide tiles would pad x by 40%
    assert (b["kernels"], b["tile_x"], b["tile_y"]) == (N.KERNELS_SPLIT, 32, 8)
    c = shape(120, 40, 40, L.Precision.FP64)  # the pair kernel is FP32 arithmetic
    assert (c["kernels"], c["tile_x"], c["tile_y"]) == (N.KERNELS_SPLIT, 32, 8)
    for s in (a, b, c):
        assert 0 < s["zchunk"] <= 40  # fixed chunks, not the balanced schedule (0)
