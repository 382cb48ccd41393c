"""NumPy restatement of the flow / order statistics (TEST INFRASTRUCTURE ONLY).

The reference has no spectrum or correlation analysis (its analysis stops at
the defect finder, src/analysis/defect_finder.tpp), so these are the
definitions the library documents in include/lbman3d.h, written with full
complex FFTs (numpy.fft) instead of the library's half-spectrum cuFFT
transforms, plus a direct-sum autocorrelation used to pin the FFT form on
small boxes.  Parity for these rows is unpinned by the reference.

Fields use the library's host layout: arrays of shape (components, V) with
cell = (z*ny + y)*nx + x.
"""
from __future__ import annotations

import math

import numpy as np


def _grid(a, nx, ny, nz):
    return np.asarray(a, dtype=np.float64).reshape(-1, nz, ny, nx)


def _kshell(nx, ny, nz):
    nmax = max(nx, ny, nz)
    mz = np.fft.fftfreq(nz) * nz
    my = np.fft.fftfreq(ny) * ny
    mx = np.fft.fftfreq(nx) * nx
    fz, fy, fx = np.meshgrid(mz / nz, my / ny, mx / nx, indexing="ij")
    return np.floor(nmax * np.sqrt(fx * fx + fy * fy + fz * fz) + 0.5).astype(np.int64)


def _rshell(nx, ny, nz):
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    dx = np.minimum(x, nx - x)
    dy = np.minimum(y, ny - y)
    dz = np.minimum(z, nz - z)
    return np.floor(np.sqrt(dx * dx + dy * dy + dz * dz) + 0.5).astype(np.int64)


def _bin(values, shells, nbins):
    s = shells.ravel()
    keep = s < nbins
    tot = np.bincount(s[keep], weights=values.ravel()[keep], minlength=nbins)[:nbins]
    cnt = np.bincount(s[keep], minlength=nbins)[:nbins].astype(np.float64)
    return tot, cnt


def velocity_spectrum(u, nx, ny, nz, nbins):
    """E[b] = (1/2V^2) sum_{k in shell b} |u_hat(k)|^2, and wavevectors per shell."""
    g = _grid(u, nx, ny, nz)
    V = nx * ny * nz
    P = sum(np.abs(np.fft.fftn(g[c])) ** 2 for c in range(3))
    tot, cnt = _bin(P, _kshell(nx, ny, nz), nbins)
    return tot * 0.5 / (V * V), cnt


def _qq_power(q, nx, ny, nz):
    g = _grid(q, nx, ny, nz)
    X, Y = np.fft.fftn(g[0]), np.fft.fftn(g[3])
    P = 2 * np.abs(X) ** 2 + 2 * np.abs(Y) ** 2 + 2 * np.real(X * np.conj(Y))
    for k in (1, 2, 4):
        P = P + 2 * np.abs(np.fft.fftn(g[k])) ** 2
    return P


def correlation_length(C):
    """First |r| where C falls below 1/e, linear between shells; -1 if never."""
    t = math.exp(-1.0)
    for b in range(1, len(C)):
        if C[b] < t:
            return (b - 1) + (C[b - 1] - t) / (C[b - 1] - C[b])
    return -1.0


def q_correlation(q, nx, ny, nz, nbins):
    """C[b] = <Q(x):Q(x+r)> / <Q:Q> averaged over |r| shells (minimum image),
    separations per shell, and the 1/e correlation length."""
    G = np.real(np.fft.ifftn(_qq_power(q, nx, ny, nz)))
    tot, cnt = _bin(G, _rshell(nx, ny, nz), nbins)
    g0 = tot[0] / cnt[0]
    C = np.where(cnt > 0, tot / np.maximum(cnt, 1) / g0, 0.0)
    return C, cnt, correlation_length(C)


def q_autocorrelation_direct(q, nx, ny, nz):
    """sum_x Q(x):Q(x+r) for every periodic separation r, by direct sums
    (small boxes only); same layout as the FFT form's real-space array."""
    g = _grid(q, nx, ny, nz)
    full = np.empty((3, 3) + g.shape[1:])
    xx, xy, xz, yy, yz = g
    zz = -(xx + yy)
    full[0, 0], full[0, 1], full[0, 2] = xx, xy, xz
    full[1, 0], full[1, 1], full[1, 2] = xy, yy, yz
    full[2, 0], full[2, 1], full[2, 2] = xz, yz, zz
    out = np.zeros(g.shape[1:])
    for rz in range(nz):
        for ry in range(ny):
            for rx in range(nx):
                sh = np.roll(full, shift=(-rz, -ry, -rx), axis=(2, 3, 4))
                out[rz, ry, rx] = np.sum(full * sh)
    return out


def speed_moments(u, V):
    u = np.asarray(u, dtype=np.float64).reshape(3, V)
    s2 = np.sum(u * u, axis=0)
    return float(np.mean(np.sqrt(s2))), float(np.mean(s2))
