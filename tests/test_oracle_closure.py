"""The closure oracle (oracle/closure.py) against finite differences.

The reference has no learned closure; the FP64 oracle network is pinned by a
central-difference check of its backpropagated gradient, and its BF16
emulation by closeness to the exact network.
"""
import numpy as np

from oracle import closure as K


def _case(grid, seed):
    nx, ny, nz = grid
    V = nx * ny * nz
    r = np.random.default_rng(seed)
    feat = r.standard_normal((9, V))
    tgt = r.standard_normal((8, V))
    p = np.zeros(K.NPARAMS)
    for (cin, cout), (w0, b0), rc, rco in zip(K.LAYERS, K.OFFSETS, (9, 32, 32, 32), (32, 32, 32, 8)):
        W = np.zeros((27, cin, cout))
        W[:, :rc, :rco] = r.standard_normal((27, rc, rco)) * np.sqrt(2.0 / (27 * rc))
        p[w0:b0] = W.ravel()
        p[b0:b0 + rco] = 0.1 * r.standard_normal(rco)
    return feat, tgt, p, np.zeros(9), np.ones(9), np.full(8, 2.0)


def test_gradient_matches_finite_differences():
    grid = (3, 4, 5)
    feat, tgt, p, sh, sc, osc = _case(grid, 1)
    loss, g = K.loss_and_grad(feat, tgt, grid, p, sh, sc, osc, bf=False)
    r = np.random.default_rng(2)
    nz = np.flatnonzero(p)
    for i in r.choice(nz, 25, replace=False):
        h = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        fp = K.loss_and_grad(feat, tgt, grid, pp, sh, sc, osc, bf=False)[0]
        fm = K.loss_and_grad(feat, tgt, grid, pm, sh, sc, osc, bf=False)[0]
        fd = (fp - fm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_bf16_emulation_is_close_to_exact():
    grid = (4, 4, 4)
    feat, tgt, p, sh, sc, osc = _case(grid, 3)
    o1, _ = K.forward(feat, grid, p, sh, sc, bf=False)
    o2, _ = K.forward(feat, grid, p, sh, sc, bf=True)
    assert np.max(np.abs(o1 - o2)) <= 0.05 * np.max(np.abs(o1))
    assert K.bf16(np.float32(1.0 + 2 ** -9)) == 1.0  # ties to even
    assert K.bf16(np.float32(1.0 + 3 * 2 ** -9)) == 1.0 + 2 ** -7
