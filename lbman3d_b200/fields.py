"""Host field containers with the reference's member names
(src/local_grid.h, src/fluid_fields.h, src/qtensor_fields.h).

Storage is numpy float64 in the reference's host layout: scalar fields
indexed by cell = (z*ny + y)*nx + x, populations AoS ``f[cell*15 + i]``
(src/local_grid.h:66).  Single-rank grids only (kHaloMPI = 0).
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from .params import Params

NDIR = 15


@dataclass
class LocalGrid:
    local_nx: int
    local_ny: int
    local_nz: int
    offset_x: int = 0
    offset_y: int = 0
    offset_z: int = 0
    kHaloMPI: int = 0

    @staticmethod
    def SingleRank(p: Params) -> "LocalGrid":
        return LocalGrid(p.nx, p.ny, p.nz)

    def idx(self, x, y, z):
        return (z * self.local_ny + y) * self.local_nx + x

    def halo_idx(self, x, y, z, i=None):
        c = self.idx(x, y, z)
        return c if i is None else c * NDIR + i

    def Volume(self):
        return self.local_nx * self.local_ny * self.local_nz

    HaloVolume = Volume


class FluidFields:
    """Populations, macroscopic fields and body force (src/fluid_fields.h:11-22)."""

    def __init__(self, grid: LocalGrid, kDensity: float = 1.0):
        V = grid.Volume()
        self.grid = grid
        self.f = np.zeros(V * NDIR)
        self.f_new = np.zeros(V * NDIR)
        self.fx, self.fy, self.fz = np.zeros(V), np.zeros(V), np.zeros(V)
        self.rho = np.full(V, kDensity)
        self.ux, self.uy, self.uz = np.zeros(V), np.zeros(V), np.zeros(V)

    def SwapFandFnew(self):
        self.f, self.f_new = self.f_new, self.f

    # layout helpers for the C ABI (3 blocks of V; populations direction-major)
    def u3(self):
        return np.concatenate([self.ux, self.uy, self.uz])

    def force3(self):
        return np.concatenate([self.fx, self.fy, self.fz])

    def f_soa(self):
        return np.ascontiguousarray(self.f.reshape(-1, NDIR).T).reshape(-1)

    def set_f_soa(self, f15):
        self.f[:] = f15.reshape(NDIR, -1).T.reshape(-1)


class QTensorFields:
    """Q components, their successors and the nematic stress
    (src/qtensor_fields.h:10-33)."""

    COMPS = ("qxx", "qxy", "qxz", "qyy", "qyz")

    def __init__(self, grid: LocalGrid):
        V = grid.Volume()
        self.grid = grid
        for c in self.COMPS:
            setattr(self, c, np.zeros(V))
            setattr(self, c + "_new", np.zeros(V))
        for c in ("Sigma_xx", "Sigma_xy", "Sigma_xz", "Sigma_yy", "Sigma_yz", "Tau_xy", "Tau_xz", "Tau_yz"):
            setattr(self, c, np.zeros(V))

    def SwapWithNew(self):
        for c in self.COMPS:
            a, b = getattr(self, c), getattr(self, c + "_new")
            setattr(self, c, b)
            setattr(self, c + "_new", a)

    def q5(self):
        return np.concatenate([getattr(self, c) for c in self.COMPS])

    def set_q5(self, q5):
        V = self.grid.Volume()
        for k, c in enumerate(self.COMPS):
            getattr(self, c)[:] = q5[k * V:(k + 1) * V]
