"""Learned closure for coarse-grid active-nematic runs (no counterpart in the
reference): a 4-layer 3x3x3 periodic CNN, trained and run on the GPU by the
library's own tcgen05 BF16 forward / backward kernels (include/lbman3d.h,
lbman_closure_*).

A coarse solver on a grid ``factor`` times coarser than the fine one takes
one step per ``factor`` fine steps (acoustic scaling: lattice velocities
unchanged); ``coarse_params`` maps the physical parameters so that both grids
solve the same continuum equations.  After every coarse step the network,
fed the state before the step, corrects Q and u.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import replace

import numpy as np

from . import _native as N
from .params import Params

PARAM_COUNT = None


def param_count() -> int:
    return int(N.lib().lbman_closure_param_count())


def coarse_params(fine: Params, factor: int) -> Params:
    """Lattice parameters of the factor-times coarser grid with dt_c = factor
    dt (acoustic scaling).  With dx -> f dx and dt -> f dt:
    nu -> nu / f (tau_c = 1/2 + (tau - 1/2) / f), Gamma -> f Gamma,
    L -> L / f^2, mu -> f mu; A, B, C, lambda and the active coefficient
    (force density ~ dt^2 / dx^2) are unchanged."""
    f = float(factor)
    return replace(fine, nx=fine.nx // factor, ny=fine.ny // factor, nz=fine.nz // factor,
                   TAUF=0.5 + (fine.TAUF - 0.5) / f, GAMMA=fine.GAMMA * f, L=fine.L / (f * f),
                   MU=fine.MU * f)


class Closure:
    """Handle on an lbman_closure (one coarse grid size)."""

    def __init__(self, nx: int, ny: int, nz: int, seed: int = 0, device: int = 0):
        h = C.c_void_p()
        N.check(N.lib().lbman_closure_create(int(device), int(nx), int(ny), int(nz), int(seed), C.byref(h)))
        self._h = h
        self.grid = (nx, ny, nz)
        self.V = nx * ny * nz

    def close(self):
        if getattr(self, "_h", None):
            try:
                N.lib().lbman_closure_destroy(self._h)
            except (AttributeError, TypeError):  # interpreter shutdown: module globals already cleared
                pass
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # --- parameters -----------------------------------------------------------
    def params(self) -> np.ndarray:
        p = np.zeros(param_count(), dtype=np.float32)
        N.check(N.lib().lbman_closure_get_params(self._h, N.fptr(p)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        N.check(N.lib().lbman_closure_set_params(self._h, N.fptr(p)))

    def scales(self):
        a, b, c = np.zeros(9, np.float32), np.zeros(9, np.float32), np.zeros(8, np.float32)
        N.check(N.lib().lbman_closure_get_scales(self._h, N.fptr(a), N.fptr(b), N.fptr(c)))
        return a, b, c

    def set_scales(self, shift, scale, out_scale):
        a, b, c = (np.ascontiguousarray(x, dtype=np.float32) for x in (shift, scale, out_scale))
        N.check(N.lib().lbman_closure_set_scales(self._h, N.fptr(a), N.fptr(b), N.fptr(c)))

    # --- network on host arrays ------------------------------------------------
    def forward(self, feat9) -> np.ndarray:
        x = np.ascontiguousarray(feat9, dtype=np.float32).reshape(9 * self.V)
        out = np.zeros(8 * self.V, dtype=np.float32)
        N.check(N.lib().lbman_closure_forward(self._h, N.fptr(x), N.fptr(out)))
        return out.reshape(8, self.V)

    def gradient(self, feat9, target8):
        x = np.ascontiguousarray(feat9, dtype=np.float32).reshape(9 * self.V)
        t = np.ascontiguousarray(target8, dtype=np.float32).reshape(8 * self.V)
        g = np.zeros(param_count(), dtype=np.float32)
        loss = C.c_double()
        N.check(N.lib().lbman_closure_gradient(self._h, N.fptr(x), N.fptr(t), C.byref(loss), N.fptr(g)))
        return loss.value, g

    # --- training set, training, corrected runs ---------------------------------
    def record(self, fine, new_trajectory: bool = False):
        N.check(N.lib().lbman_closure_record(self._h, fine.handle, int(bool(new_trajectory))))

    def record_box(self, ensemble, box: int, trajectory: int):
        """Snapshot of ensemble box `box` as trajectory `trajectory`."""
        N.check(N.lib().lbman_closure_record_box(self._h, ensemble._h, int(box), int(trajectory)))

    def add_rollout_pairs(self, coarse, m: int, stride: int = 1) -> int:
        """Pairs from m-step corrected runs (lbman_closure_add_rollout_pairs)."""
        n = C.c_int()
        N.check(N.lib().lbman_closure_add_rollout_pairs(self._h, coarse.handle, int(m), int(stride), C.byref(n)))
        return n.value

    def dataset(self):
        a, b = C.c_int(), C.c_int()
        N.check(N.lib().lbman_closure_dataset(self._h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def build_targets(self, coarse, fit_scales: bool = True):
        N.check(N.lib().lbman_closure_build_targets(self._h, coarse.handle, int(bool(fit_scales))))

    def train(self, iters: int, lr: float = 1e-3, seed: int = 0):
        a, b = C.c_double(), C.c_double()
        N.check(N.lib().lbman_closure_train(self._h, int(iters), float(lr), int(seed), C.byref(a), C.byref(b)))
        return a.value, b.value

    def load_snapshot(self, k: int, coarse):
        N.check(N.lib().lbman_closure_load_snapshot(self._h, int(k), coarse.handle))

    def set_options(self, train_noise: float = 0.0, gain: float = 1.0):
        """Input noise (std, normalised units) in training; correction gain."""
        N.check(N.lib().lbman_closure_set_options(self._h, float(train_noise), float(gain)))

    def set_wait_limit(self, polls: int = None):
        """Polls of each tensor-core completion wait before it gives up
        (None: the default); a wait that gives up makes the call raise with
        status LBMAN_ERR_TIMEOUT, and the next call runs normally."""
        polls = N.CLOSURE_WAIT_DEFAULT if polls is None else int(polls)
        N.check(N.lib().lbman_closure_set_wait_limit(self._h, polls))

    def step(self, coarse, n: int = 1):
        N.check(N.lib().lbman_closure_step(self._h, coarse.handle, int(n)))
