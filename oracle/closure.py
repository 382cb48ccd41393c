"""NumPy FP64 restatement of the closure network (TEST INFRASTRUCTURE ONLY).

The reference has no learned closure; this is the definition the library
documents in include/lbman3d.h (lbman_closure_*), written as explicit
periodic convolutions with np.roll, used to check the tensor-core forward
and backward passes.  With ``bf16=True`` the operands are rounded to BF16 at
the points where the CUDA kernels store BF16 (inputs, weights, activations,
pre-activations, gradients), so the remaining difference is FP32-vs-FP64
accumulation; with ``bf16=False`` it is the exact FP64 network.

Parameter vector layout (one FP32 vector): per layer W[27][cin][cout] then
b[cout], cin = 16, 32, 32, 32 and cout = 32, 32, 32, 16 (padding held at 0);
tap = (dz+1)*9 + (dy+1)*3 + (dx+1); output cell c reads input c + (dx,dy,dz).
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

LAYERS = [(16, 32), (32, 32), (32, 32), (32, 16)]
TAPS = [(t % 3 - 1, (t // 3) % 3 - 1, t // 9 - 1) for t in range(27)]  # (dx, dy, dz)


def offsets():
    off, o = [], 0
    for cin, cout in LAYERS:
        off.append((o, o + 27 * cin * cout))
        o += 27 * cin * cout + cout
    return off, o


OFFSETS, NPARAMS = offsets()


def bf16(a):
    """Round float32 values to BF16 (round to nearest even), as float64."""
    a = np.asarray(a, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32).astype(np.float64)


def unpack(params):
    p = np.asarray(params, dtype=np.float64)
    out = []
    for (cin, cout), (w0, b0) in zip(LAYERS, OFFSETS):
        out.append((p[w0:b0].reshape(27, cin, cout), p[b0:b0 + cout]))
    return out


def gelu(x):
    return 0.5 * x * (1.0 + erf(x / np.sqrt(2.0)))


def gelu_grad(x):
    return 0.5 * (1.0 + erf(x / np.sqrt(2.0))) + x * np.exp(-0.5 * x * x) / np.sqrt(2.0 * np.pi)


def _shift(a, dx, dy, dz):
    """a[z+dz, y+dy, x+dx] (periodic) for a of shape (nz, ny, nx, C)."""
    return np.roll(a, shift=(-dz, -dy, -dx), axis=(0, 1, 2))


def conv(a, W):
    out = 0.0
    for t, (dx, dy, dz) in enumerate(TAPS):
        out = out + np.einsum("zyxi,io->zyxo", _shift(a, dx, dy, dz), W[t])
    return out


def conv_input_grad(g, W):
    out = 0.0
    for t, (dx, dy, dz) in enumerate(TAPS):
        out = out + np.einsum("zyxo,io->zyxi", _shift(g, -dx, -dy, -dz), W[t])
    return out


def conv_weight_grad(a, g):
    return np.stack([np.einsum("zyxi,zyxo->io", _shift(a, dx, dy, dz), g) for (dx, dy, dz) in TAPS])


def features(feat9, grid, shift, scale):
    nx, ny, nz = grid
    x = np.asarray(feat9, dtype=np.float64).reshape(9, nz, ny, nx)
    a = np.zeros((nz, ny, nx, 16))
    for j in range(9):
        a[..., j] = (x[j] - shift[j]) / scale[j]
    return a


def forward(feat9, grid, params, shift, scale, bf=True):
    """Network outputs (nz, ny, nx, 16) and the cached activations."""
    r = bf16 if bf else (lambda v: np.asarray(v, dtype=np.float64))
    layers = unpack(params)
    a = r(features(feat9, grid, shift, scale))
    cache = {"a": [a], "pre": []}
    for li, (W, b) in enumerate(layers):
        p = conv(a, r(W)) + b
        if li < 3:
            cache["pre"].append(r(p))
            a = r(gelu(p))
            cache["a"].append(a)
        else:
            out = p
    return out, cache


def loss_and_grad(feat9, target8, grid, params, shift, scale, out_scale, bf=True):
    """(loss, flat gradient) of (1/8V) sum (out_j - target_j/out_scale_j)^2."""
    r = bf16 if bf else (lambda v: np.asarray(v, dtype=np.float64))
    nx, ny, nz = grid
    V = nx * ny * nz
    layers = unpack(params)
    out, cache = forward(feat9, grid, params, shift, scale, bf)
    t = np.asarray(target8, dtype=np.float64).reshape(8, nz, ny, nx)
    d = np.zeros_like(out)
    for j in range(8):
        d[..., j] = out[..., j] - t[j] / out_scale[j]
    loss = float(np.sum(d[..., :8] ** 2) / (8 * V))
    g = r(2.0 * d / (8 * V))
    g[..., 8:] = 0.0
    grad = np.zeros(NPARAMS)
    for li in range(3, -1, -1):
        W, _ = layers[li]
        (w0, b0) = OFFSETS[li]
        cin, cout = LAYERS[li]
        grad[w0:b0] = conv_weight_grad(cache["a"][li], g).ravel()
        grad[b0:b0 + cout] = g.reshape(-1, cout).sum(axis=0)
        if li > 0:
            g = r(conv_input_grad(g, r(W)) * gelu_grad(cache["pre"][li - 1]))
    return loss, grad
