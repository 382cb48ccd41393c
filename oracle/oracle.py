"""ctypes wrapper of oracle/lbman_oracle.c -- the CPU restatement of the
reference's per-timestep path.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline leg as the checker.  Nothing in lbman3d_b200/ imports
it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "lbman_oracle.c")
LIB = os.path.join(HERE, "liblbman_oracle.so")

Q_PERIODIC, Q_NEUMANN, Q_ANCHORING = 0, 1, 2
U_PERIODIC, U_NOSLIP, U_MOVING, U_SPECULAR = 0, 1, 2, 3
CENTRED, UPWIND = 0, 1


class Face(C.Structure):
    _fields_ = [("qbc", C.c_int), ("s", C.c_double), ("theta", C.c_double), ("phi", C.c_double),
                ("ubc", C.c_int), ("uw", C.c_double * 3)]


class Params(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("DT", C.c_double), ("kDensity", C.c_double), ("TAUF", C.c_double),
                ("L", C.c_double), ("A", C.c_double), ("B", C.c_double), ("C", C.c_double),
                ("LAMBDA", C.c_double), ("GAMMA", C.c_double), ("ALPHA", C.c_double),
                ("MU", C.c_double), ("advection", C.c_int), ("face", Face * 6)]


def build(force: bool = False) -> str:
    """Compile the restatement (gcc, no FMA contraction) if it is stale."""
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(
            os.path.getmtime(SRC), os.path.getmtime(os.path.join(HERE, "lbman_oracle.h"))):
        subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-ffp-contract=off", "-fno-fast-math",
                        "-fopenmp", "-o", LIB, SRC, "-lm"], check=True)
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        dp = C.POINTER(C.c_double)
        L.orc_params_default.argtypes = [C.POINTER(Params)]
        L.orc_anchored_q.argtypes = [C.POINTER(Face), dp]
        L.orc_equilibrium_order.argtypes = [C.POINTER(Params)]
        L.orc_equilibrium_order.restype = C.c_double
        L.orc_new.argtypes = [C.POINTER(Params)]
        L.orc_new.restype = C.c_void_p
        L.orc_free.argtypes = [C.c_void_p]
        L.orc_set.argtypes = [C.c_void_p, dp, dp, dp, dp, dp]
        L.orc_get.argtypes = [C.c_void_p, dp, dp, dp, dp, dp, dp, dp]
        L.orc_step.argtypes = [C.c_void_p, C.c_int]
        L.orc_q_step.argtypes = [C.c_void_p, C.c_int]
        L.orc_lbm_step.argtypes = [C.c_void_p]
        L.orc_free_energy.argtypes = [C.POINTER(Params), dp]
        L.orc_free_energy.restype = C.c_double
        L.orc_log_reduce.argtypes = [C.POINTER(Params), dp, dp, dp, dp]
        L.orc_order_director.argtypes = [C.POINTER(Params), dp, dp, dp]
        u8p = C.POINTER(C.c_uint8)
        L.orc_winding.argtypes = [C.POINTER(Params), dp, u8p, u8p, u8p]
        L.orc_winding.restype = C.c_int64
        L.orc_seeded_q.argtypes = [C.POINTER(Params), C.c_uint64, C.c_double, C.c_double, dp]
        _lib = L
    return _lib


def _dp(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


def make_params(nx, ny, nz, faces, advection=CENTRED, **phys) -> Params:
    """faces: 6 tuples (qbc, (s, theta, phi), ubc, (ux, uy, uz)) in XLo..ZHi order."""
    p = Params()
    lib().orc_params_default(C.byref(p))
    p.nx, p.ny, p.nz = nx, ny, nz
    p.advection = advection
    for k, v in phys.items():
        setattr(p, k, v)
    for k, (qbc, anc, ubc, uw) in enumerate(faces):
        p.face[k].qbc = qbc
        p.face[k].s, p.face[k].theta, p.face[k].phi = anc
        p.face[k].ubc = ubc
        for j in range(3):
            p.face[k].uw[j] = uw[j]
    return p


class OracleSim:
    """A CPU simulation state (fields live inside the C library)."""

    def __init__(self, params: Params):
        self.p = params
        self.V = params.nx * params.ny * params.nz
        self.h = lib().orc_new(C.byref(params))
        if not self.h:
            raise MemoryError("orc_new failed")

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_free(self.h)
            self.h = None

    def set(self, rho, u, q, f=None, force=None):
        c = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
        rho, u, q, f, force = c(rho), c(u), c(q), c(f), c(force)
        lib().orc_set(self.h, _dp(rho), _dp(u), _dp(q), _dp(f), _dp(force))

    def get(self):
        V = self.V
        out = dict(rho=np.empty(V), u=np.empty(3 * V), q=np.empty(5 * V), f=np.empty(15 * V),
                   force=np.empty(3 * V), sigma=np.empty(5 * V), tau=np.empty(3 * V))
        lib().orc_get(self.h, *[_dp(out[k]) for k in ("rho", "u", "q", "f", "force", "sigma", "tau")])
        return out

    def step(self, n=1):
        lib().orc_step(self.h, n)

    def q_step(self, with_active=True):
        lib().orc_q_step(self.h, 1 if with_active else 0)

    def lbm_step(self):
        lib().orc_lbm_step(self.h)


def free_energy(p: Params, q) -> float:
    q = np.ascontiguousarray(q, dtype=np.float64)
    return lib().orc_free_energy(C.byref(p), _dp(q))


def log_reduce(p: Params, rho, u, upast):
    out = np.zeros(8)
    lib().orc_log_reduce(C.byref(p), _dp(np.ascontiguousarray(rho)), _dp(np.ascontiguousarray(u)),
                         _dp(upast), _dp(out))
    return out


def order_director(p: Params, q):
    V = p.nx * p.ny * p.nz
    S, d = np.empty(V), np.empty(3 * V)
    lib().orc_order_director(C.byref(p), _dp(np.ascontiguousarray(q)), _dp(S), _dp(d))
    return S, d


def winding(p: Params, director):
    nx, ny, nz = p.nx, p.ny, p.nz
    dx = np.zeros(max(nx * (ny - 1) * (nz - 1), 1), np.uint8)
    dy = np.zeros(max((nx - 1) * ny * (nz - 1), 1), np.uint8)
    dz = np.zeros(max((nx - 1) * (ny - 1) * nz, 1), np.uint8)
    u8 = lambda a: a.ctypes.data_as(C.POINTER(C.c_uint8))
    n = lib().orc_winding(C.byref(p), _dp(np.ascontiguousarray(director)), u8(dx), u8(dy), u8(dz))
    return int(n), dx, dy, dz


def seeded_q(p: Params, seed: int, S0: float, sigma: float):
    q = np.empty(5 * p.nx * p.ny * p.nz)
    lib().orc_seeded_q(C.byref(p), seed, S0, sigma, _dp(q))
    return q


def equilibrium_order(p: Params) -> float:
    return lib().orc_equilibrium_order(C.byref(p))
