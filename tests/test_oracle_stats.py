"""The statistics oracle (oracle/stats.py) against direct definitions.

The reference has no spectrum or correlation analysis, so these pins are
analytic: the FFT autocorrelation equals the direct periodic sum, the
spectrum obeys Parseval and puts a single Fourier mode in its one shell.
"""
import math

import numpy as np

from oracle import stats as S


def _rand(shape, seed):
    return np.random.default_rng(seed).standard_normal(shape)


def test_autocorrelation_fft_equals_direct_sum():
    nx, ny, nz = 4, 5, 6
    q = _rand((5, nx * ny * nz), 1)
    direct = S.q_autocorrelation_direct(q, nx, ny, nz)
    fft = np.real(np.fft.ifftn(S._qq_power(q, nx, ny, nz)))
    np.testing.assert_allclose(fft, direct, rtol=1e-12, atol=1e-10)


def test_spectrum_parseval_and_single_mode():
    nx, ny, nz = 6, 8, 10
    V = nx * ny * nz
    u = _rand((3, V), 2)
    E, cnt = S.velocity_spectrum(u, nx, ny, nz, 20)
    assert math.isclose(E.sum(), 0.5 * np.mean(np.sum(u * u, axis=0)), rel_tol=1e-12)
    assert cnt.sum() == V
    # u_x = A sin(2 pi m y / ny): all energy A^2/4 in shell round(nmax m / ny)
    A, m = 0.3, 2
    y = np.arange(ny)
    ux = np.broadcast_to(A * np.sin(2 * np.pi * m * y / ny)[None, :, None], (nz, ny, nx)).ravel()
    u1 = np.stack([ux, np.zeros(V), np.zeros(V)])
    E1, _ = S.velocity_spectrum(u1, nx, ny, nz, 20)
    b = int(math.floor(max(nx, ny, nz) * m / ny + 0.5))
    assert math.isclose(E1[b], A * A / 4, rel_tol=1e-12)
    assert abs(E1.sum() - E1[b]) < 1e-14


def test_correlation_uniform_and_length():
    nx = ny = nz = 8
    V = nx * ny * nz
    q = np.zeros((5, V))
    q[0] = -0.1
    q[3] = -0.1
    C, cnt, xi = S.q_correlation(q, nx, ny, nz, 8)
    np.testing.assert_allclose(C[cnt > 0], 1.0, rtol=1e-12)
    assert xi == -1.0
    assert S.correlation_length([1.0, 0.5, 0.2]) == 1.0 + (0.5 - math.exp(-1)) / 0.3
