"""Boundary-condition tags, WallSpec and presets: the run-time form of the
reference's src/boundary.h and src/sim_config.h.

The reference selects boundary behaviour through types
(``WallSpec<Neumann, NoSlip>``, ``Anchoring<S, theta, phi>``,
``MovingWall<Ux, Uy, Uz>``); here the same names are small value objects and
a configuration is lowered to six face descriptors for the C ABI.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

from . import _native as N


class _Tag:
    def __repr__(self):
        return type(self).__name__ + "()"

    def __eq__(self, other):
        return type(self) is type(other) and vars(self) == vars(other)

    def __hash__(self):
        return hash((type(self).__name__,) + tuple(sorted(vars(self).items())))


class Periodic(_Tag):
    """Periodic stencil / periodic streaming (src/boundary.h:31)."""


class Neumann(_Tag):
    """Zero-flux Q stencil: ghost equals the boundary value (src/boundary.h:32)."""


class NoSlip(_Tag):
    """Mid-point bounce-back, u_wall = 0 (src/boundary.h:33)."""


class SpecularReflection(_Tag):
    """Mirror reflection: free slip, no penetration (src/boundary.h:34)."""


class Anchoring(_Tag):
    """Strong anchoring at order S and director angles (theta, phi) in radians
    (src/boundary.h:37-42)."""

    def __init__(self, S: float = 1.0, theta: float = 0.0, phi: float = 0.0):
        self.s, self.theta, self.phi = float(S), float(theta), float(phi)

    def __repr__(self):
        return f"Anchoring({self.s}, {self.theta}, {self.phi})"


class MovingWall(_Tag):
    """Bounce-back with an imposed wall velocity (src/boundary.h:45-50)."""

    def __init__(self, Ux: float = 0.0, Uy: float = 0.0, Uz: float = 0.0):
        self.Ux, self.Uy, self.Uz = float(Ux), float(Uy), float(Uz)

    def __repr__(self):
        return f"MovingWall({self.Ux}, {self.Uy}, {self.Uz})"


@dataclass(frozen=True)
class WallSpec:
    """Q stencil policy + velocity BC for one face (src/boundary.h:72-76)."""
    QBC: _Tag
    UBC: _Tag

    def lower(self) -> N.lbman_face:
        f = N.lbman_face()
        q, u = self.QBC, self.UBC
        if isinstance(q, Periodic):
            f.qbc = N.Q_PERIODIC
        elif isinstance(q, Neumann):
            f.qbc = N.Q_NEUMANN
        elif isinstance(q, Anchoring):
            f.qbc = N.Q_ANCHORING
            f.s, f.theta, f.phi = q.s, q.theta, q.phi
        else:
            raise TypeError(f"not a Q boundary tag: {q!r}")
        if isinstance(u, Periodic):
            f.ubc = N.U_PERIODIC
        elif isinstance(u, NoSlip):
            f.ubc = N.U_NOSLIP
        elif isinstance(u, MovingWall):
            f.ubc = N.U_MOVING
            f.uw[0], f.uw[1], f.uw[2] = u.Ux, u.Uy, u.Uz
        elif isinstance(u, SpecularReflection):
            f.ubc = N.U_SPECULAR
        else:
            raise TypeError(f"not a velocity boundary tag: {u!r}")
        return f


FACES = ("XLo", "XHi", "YLo", "YHi", "ZLo", "ZHi")
_NEU_NOSLIP = WallSpec(Neumann(), NoSlip())
_PER = WallSpec(Periodic(), Periodic())


class BCConfig:
    """Six independently specified faces (src/boundary.h:84-100).  Defaults to
    WallSpec<Neumann, NoSlip> on every face, as the reference template does."""
    name = "Custom"

    def __init__(self, XLo=_NEU_NOSLIP, XHi=_NEU_NOSLIP, YLo=_NEU_NOSLIP, YHi=_NEU_NOSLIP,
                 ZLo=_NEU_NOSLIP, ZHi=_NEU_NOSLIP, name: str | None = None):
        self.XLo, self.XHi, self.YLo, self.YHi, self.ZLo, self.ZHi = XLo, XHi, YLo, YHi, ZLo, ZHi
        if name:
            self.name = name

    def faces(self):
        return [getattr(self, k) for k in FACES]

    def __repr__(self):
        return f"{type(self).__name__}(" + ", ".join(f"{k}={getattr(self, k)}" for k in FACES) + ")"


class FullyPeriodicConfig(BCConfig):
    """All faces periodic (src/boundary.h:105-113)."""
    name = "FullyPeriodic"

    def __init__(self):
        super().__init__(*([_PER] * 6))


class ChannelConfig(BCConfig):
    """No-slip Neumann walls on X and Y, periodic Z (src/boundary.h:116-124)."""
    name = "Channel"

    def __init__(self):
        super().__init__(_NEU_NOSLIP, _NEU_NOSLIP, _NEU_NOSLIP, _NEU_NOSLIP, _PER, _PER)


class SlitConfig(BCConfig):
    """Free-slip (specular) plates confining X (src/sim_config.h:19-27)."""
    name = "SlitFreeSlip"

    def __init__(self):
        w = WallSpec(Neumann(), SpecularReflection())
        super().__init__(w, w, _PER, _PER, _PER, _PER)


class SlitNoSlipConfig(BCConfig):
    """No-slip plates confining X (src/sim_config.h:37-45)."""
    name = "SlitNoSlip"

    def __init__(self):
        super().__init__(_NEU_NOSLIP, _NEU_NOSLIP, _PER, _PER, _PER, _PER)


PeriodicBC = FullyPeriodicConfig  # backward-compatible alias (src/boundary.h:134)
SimBC = SlitNoSlipConfig          # the reference's default selection (src/sim_config.h:48)


def periodicity_by_axis(bc: BCConfig):
    """(src/boundary.h:131-136)"""
    return [int(isinstance(getattr(bc, f).UBC, Periodic)) for f in ("XLo", "YLo", "ZLo")]


def is_wall_by_face(bc: BCConfig):
    """(src/boundary.h:141-148)"""
    return [not isinstance(w.UBC, Periodic) for w in bc.faces()]


def from_face_tuples(faces, name="Custom") -> BCConfig:
    """Build a BCConfig from (qbc, (S, theta, phi), ubc, (Ux, Uy, Uz)) tuples
    with integer tags (the form used by the parity fixtures)."""
    specs = []
    for qbc, anc, ubc, uw in faces:
        q = [Periodic(), Neumann(), Anchoring(*anc)][qbc]
        u = [Periodic(), NoSlip(), MovingWall(*uw), SpecularReflection()][ubc]
        specs.append(WallSpec(q, u))
    return BCConfig(*specs, name=name)


def anchored_q(a: Anchoring):
    """AnchoredQ (src/boundary_handler.h:232-251): the 5 stored components."""
    sin_sq_phi = 0.5 * (1.0 - math.cos(2.0 * a.phi))
    cos_sq_phi = 1.0 - sin_sq_phi
    sin_phi_cos_phi = 0.5 * math.sin(2.0 * a.phi)
    sin_sq_th = 0.5 * (1.0 - math.cos(2.0 * a.theta))
    sin_th_cos_th = 0.5 * math.sin(2.0 * a.theta)
    S = a.s
    return (S * (cos_sq_phi * sin_sq_th - 1.0 / 3.0), S * (sin_phi_cos_phi * sin_sq_th),
            S * (math.cos(a.phi) * sin_th_cos_th), S * (sin_sq_phi * sin_sq_th - 1.0 / 3.0),
            S * (math.sin(a.phi) * sin_th_cos_th))
