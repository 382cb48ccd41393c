"""The learned closure on the GPU: the tcgen05 self-test, forward and
gradient against the FP64 oracle network (oracle/closure.py) with BF16
emulation, and the record -> targets -> train -> corrected-run pipeline.
Parity for this row is unpinned by the reference (it has no closure).
"""
import numpy as np
import pytest

import lbman3d_b200 as L
from lbman3d_b200 import _native as N
from lbman3d_b200 import closure as CL
from oracle import closure as K

pytestmark = pytest.mark.gpu


def _case(grid, seed):
    nx, ny, nz = grid
    V = nx * ny * nz
    r = np.random.default_rng(seed)
    feat = r.standard_normal((9, V)).astype(np.float32)
    feat[0] += 1.0
    tgt = r.standard_normal((8, V)).astype(np.float32)
    return feat, tgt


def test_tensor_core_selftest():
    e = np.zeros(4)
    L._native.check(L._native.lib().lbman_closure_selftest(0, L._native.dptr(e)))
    assert np.all(e >= 0) and np.all(e < 1e-6), e


# (8, 8, 8), (5, 6, 7): gathers from global memory; (64, 4, 4): 128-cell
# tiles of whole x rows, staged through shared memory; (16, 16, 8), (32, 64,
# 40): the z-marching descriptor-halo kernel (one plane per block, and 16
# columns marching 3-plane ranges with a shorter last range)
@pytest.mark.parametrize("grid", [(8, 8, 8), (5, 6, 7), (16, 16, 8), (64, 4, 4), (32, 64, 40)])
def test_forward_matches_oracle(grid):
    feat, _ = _case(grid, 1)
    with CL.Closure(*grid, seed=5) as cl:
        p = cl.params()
        sh, sc, _ = cl.scales()
        got = cl.forward(feat)
    ref, _ = K.forward(feat, grid, p, sh, sc, bf=True)
    ref = ref[..., :8].reshape(-1, 8).T
    assert np.max(np.abs(got - ref)) <= 2e-2 * np.max(np.abs(ref))


# (8, 8, 8): the gather convolution and weight-gradient kernels; (16, 16, 8):
# the descriptor-halo forms.  A limit of 0 polls makes the first completion
# wait of every CTA give up while its MMAs still run to completion, so the
# timeout path is exercised without a fault: the call must report
# LBMAN_ERR_TIMEOUT, and the next call at the default limit must give the
# same outputs and gradients as before.
@pytest.mark.parametrize("grid", [(8, 8, 8), (16, 16, 8)])
def test_wait_that_gives_up_reports_timeout_and_next_call_recovers(grid):
    feat, tgt = _case(grid, 3)
    with CL.Closure(*grid, seed=7) as cl:
        out0 = cl.forward(feat)
        loss0, g0 = cl.gradient(feat, tgt)
        cl.set_wait_limit(0)
        for call in (lambda: cl.forward(feat), lambda: cl.gradient(feat, tgt)):
            with pytest.raises(L._native.LbmanError) as e:
                call()
            assert e.value.status == L._native.ERR_TIMEOUT
        cl.set_wait_limit()
        np.testing.assert_array_equal(cl.forward(feat), out0)
        loss1, g1 = cl.gradient(feat, tgt)
        assert loss1 == loss0
        np.testing.assert_array_equal(g1, g0)


@pytest.mark.parametrize("grid", [(8, 8, 8), (5, 6, 7), (16, 16, 8), (32, 64, 40)])
def test_gradient_matches_oracle(grid):
    feat, tgt = _case(grid, 2)
    with CL.Closure(*grid, seed=6) as cl:
        p = cl.params()
        sh, sc, osc = cl.scales()
        loss, g = cl.gradient(feat, tgt)
    lref, gref = K.loss_and_grad(feat, tgt, grid, p, sh, sc, osc, bf=True)
    assert abs(loss - lref) <= 1e-3 * lref
    for (w0, b0), (cin, cout) in zip(K.OFFSETS, K.LAYERS):
        for a, b in ((w0, b0), (b0, b0 + cout)):
            x, y = g[a:b].astype(np.float64), gref[a:b]
            rel = np.linalg.norm(x - y) / max(np.linalg.norm(y), 1e-30)
            cos = x @ y / max(np.linalg.norm(x) * np.linalg.norm(y), 1e-30)
            assert rel <= 3e-2 and cos >= 0.999, (a, b, rel, cos)


def test_pipeline_trains_and_runs():
    fine_p = L.Params(nx=32, ny=32, nz=32, ALPHA=0.01)
    coarse_p = CL.coarse_params(fine_p, 4)
    assert coarse_p.nx == 8 and abs(coarse_p.TAUF - 1.0) < 1e-12
    with L.Simulation(fine_p, L.FullyPeriodicConfig(), L.Precision.FP32) as fine, \
            L.Simulation(coarse_p, L.FullyPeriodicConfig(), L.Precision.FP32) as coarse, \
            CL.Closure(8, 8, 8, seed=1) as cl:
        fine.init_seeded(3, 0.5, 1e-3)
        fine.step(40)
        cl.record(fine, new_trajectory=True)
        for _ in range(12):
            fine.step(4)
            cl.record(fine)
        assert cl.dataset() == (13, 0)
        cl.build_targets(coarse)
        assert cl.dataset() == (13, 12)
        first, last = cl.train(300, lr=1e-3, seed=2)
        assert last < 0.7 * first, (first, last)
        cl.load_snapshot(0, coarse)
        cl.step(coarse, 3)
        out = coarse.download()
        assert np.all(np.isfinite(out["q"])) and np.all(np.isfinite(out["u"]))


def test_ensemble_snapshots_and_rollout_pairs():
    """Snapshots recorded from ensemble boxes equal those of the same runs
    done alone; interleaved recordings pair within each trajectory; rollout
    pairs are added from every eligible snapshot and train."""
    fine_p = L.Params(nx=32, ny=32, nz=32, ALPHA=0.01)
    coarse_p = CL.coarse_params(fine_p, 4)
    S0 = L.EquilibriumScalarOrder(fine_p)
    seeds = [3, 4]
    with L.Ensemble([(fine_p, L.FullyPeriodicConfig())] * 2, L.Precision.FP32, N.KERNELS_SPLIT) as ens, \
            L.Simulation(fine_p, L.FullyPeriodicConfig(), L.Precision.FP32, N.KERNELS_SPLIT, tile=(32, 6, 0)) as fine, \
            L.Simulation(coarse_p, L.FullyPeriodicConfig(), L.Precision.FP32) as coarse, \
            L.Simulation(coarse_p, L.FullyPeriodicConfig(), L.Precision.FP32) as probe, \
            CL.Closure(8, 8, 8, seed=1) as cl, CL.Closure(8, 8, 8, seed=1) as ref:
        ens.set_shape(N.KERNELS_SPLIT, 32, 6, 0)  # the single box's shape: the same arithmetic
        ens.init_seeded_each(seeds, 1e-3)
        ens.step(20)
        for b in range(2):
            cl.record_box(ens, b, b)
        for _ in range(6):
            ens.step(4)
            for b in range(2):
                cl.record_box(ens, b, b)
        assert cl.dataset() == (14, 0)
        fine.init_seeded(seeds[1], S0, 1e-3)
        fine.step(20)
        ref.record(fine, new_trajectory=True)
        for _ in range(6):
            fine.step(4)
            ref.record(fine)
        # box 1's snapshots are the odd recordings
        for k in range(7):
            cl.load_snapshot(2 * k + 1, coarse)
            ref.load_snapshot(k, probe)
            a, b = coarse.download(), probe.download()
            for f in ("rho", "u", "q"):
                np.testing.assert_array_equal(a[f], b[f])
        cl.build_targets(coarse)
        assert cl.dataset() == (14, 12)  # 6 pairs per trajectory, none across them
        first, last = cl.train(200, lr=1e-3, seed=2)
        assert last < first
        # m = 2: snapshots with a third later recording of their trajectory,
        # 4 per trajectory, every one of them (stride 1)
        assert cl.add_rollout_pairs(coarse, 2, 1) == 8
        assert cl.dataset() == (14, 20)
        # m = 3: 3 eligible per trajectory, 6 in recording order, every other one
        assert cl.add_rollout_pairs(coarse, 3, 2) == 3
        cl.train(100, lr=5e-4, seed=3)
        cl.build_targets(coarse, fit_scales=False)  # clears the rollout pairs
        assert cl.dataset() == (14, 12)


def test_trained_closure_beats_plain_coarse_on_held_out_run():
    """What the network gains: after training on two seeds, one corrected
    coarse step from a held-out filtered state is closer to the filtered
    fine state than the plain coarse step, for Q and for u."""
    from lbman3d_b200 import closure_experiment as X
    r = X.run(fine_n=64, factor=4, zeta=0.01, train_seeds=(21, 22), test_seed=77, burn=200, snaps=20,
              iters=300, lr=1e-3, rollout=6, log=lambda m: None)
    first = r["short_time_relative_l2"][0]
    assert first["step"] == 1
    assert first["closure_q"] < first["plain_q"], first
    assert first["closure_u"] < first["plain_u"], first
    assert r["train"]["loss_last_tenth"] < r["train"]["loss_first_tenth"]
    assert r["cost"]["closure_ms_per_coarse_step"] > 0
