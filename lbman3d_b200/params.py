"""Run-time form of the reference's compile-time ``namespace Params``
(src/params.h) and ``sim_config.h`` choices.

Field names are the reference's; derived constants (omega, omega_prime,
omega_forcing, kinematicViscosity) are computed with the same expressions
(src/params.h:52-54, 152).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field, replace

from . import _native as N

kCs2Inv = 3.0
kCs2InvTimes2 = 6.0
kCs4Inv = 9.0
khalfCs2Inv = 1.5
khalfCs4Inv = 4.5


class Advection:
    """Finite-difference scheme of u.grad(Q) (src/qtensor_types.h:19)."""
    Centred = N.CENTRED
    Upwind = N.UPWIND


class Precision:
    FP64 = N.FP64   # the reference's arithmetic, bitwise
    FP32 = N.FP32   # FP32 compute, populations stored as f_i - w_i*rho0
    FP16 = N.FP16   # FP32 compute, FP16 deviation storage


@dataclass
class Params:
    nx: int = 20
    ny: int = 100
    nz: int = 100
    DT: float = 1.0
    kDensity: float = 1.0
    TAUF: float = 2.5
    L: float = 0.06
    A: float = 0.0
    B: float = -0.3
    C: float = 0.3
    LAMBDA: float = 0.3
    GAMMA: float = 0.34
    ALPHA: float = 0.023
    MU: float = 0.0
    NOISE: float = 0.05
    kQAdvection: int = Advection.Centred

    @property
    def omega(self):
        return 1.0 - self.DT / self.TAUF

    @property
    def omega_prime(self):
        return self.DT / self.TAUF

    @property
    def omega_forcing(self):
        return 1.0 - self.DT / 2.0 / self.TAUF

    @property
    def kinematicViscosity(self):
        return self.kDensity / kCs2Inv * (self.TAUF - 0.5 * self.DT)

    @property
    def V(self):
        return self.nx * self.ny * self.nz

    def with_(self, **kw) -> "Params":
        return replace(self, **kw)


def EquilibriumScalarOrder(p: Params) -> float:
    """Ordered root of the bulk Landau-de Gennes field (src/model.h:39-41)."""
    return (-p.B + math.sqrt(p.B * p.B - 24.0 * p.A * p.C)) / (4.0 * p.C)
