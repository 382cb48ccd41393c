"""CPU-side checks of the C ABI library and the host layer (no GPU needed):
the shared library loads and exports every entry point include/*.h
declares, configuration defaults equal params.h, invalid configurations are
rejected before any CUDA call, and the reference's BC presets lower to the
expected face descriptors."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import lbman3d_b200 as L
from lbman3d_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if fn.endswith(".h"):
            src = open(os.path.join(inc, fn)).read()
            names |= set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(lbman_[a-z_0-9]+)\s*\(", src, re.M))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = N.lib()
    decl = declared_functions()
    assert len(decl) >= 18
    for name in decl:
        assert hasattr(lib, name), name
    assert {p[0] for p in N.PROTOTYPES} >= set(decl)


def test_abi_version_and_status_strings():
    assert N.lib().lbman_abi_version() == 1
    assert N.lib().lbman_status_string(N.ERR_DIVERGED).decode().startswith("simulation diverged")


def test_config_defaults_are_params_h():
    cfg = N.lbman_config()
    assert N.lib().lbman_config_init(C.byref(cfg)) == N.OK
    p = L.Params()
    for k in ("nx", "ny", "nz", "DT", "kDensity", "TAUF", "L", "A", "B", "C", "LAMBDA", "GAMMA", "ALPHA", "MU"):
        assert getattr(cfg, k) == getattr(p, k), k
    # SimBC = SlitNoSlipConfig
    assert [cfg.face[k].ubc for k in range(6)] == [N.U_NOSLIP, N.U_NOSLIP] + [N.U_PERIODIC] * 4
    assert [cfg.face[k].qbc for k in range(6)] == [N.Q_NEUMANN, N.Q_NEUMANN] + [N.Q_PERIODIC] * 4


def _create(cfg):
    h = C.c_void_p()
    return N.lib().lbman_create(C.byref(cfg), C.byref(h)), h


def test_mixed_periodic_velocity_axis_is_rejected():
    p = L.Params(nx=8, ny=8, nz=8)
    bc = L.BCConfig(L.WallSpec(L.Periodic(), L.Periodic()), L.WallSpec(L.Neumann(), L.NoSlip()),
                    *([L.WallSpec(L.Periodic(), L.Periodic())] * 4))
    st, h = _create(L.make_config(p, bc))
    assert st == N.ERR_ARG and not h.value
    assert "periodic on one face only" in N.lib().lbman_last_error().decode()


@pytest.mark.parametrize("field,value", [("precision", 7), ("advection", 3), ("nx", 0), ("TAUF", 0.0),
                                         ("kernels", 9), ("threads", -1)])
def test_invalid_configurations_are_rejected(field, value):
    cfg = L.make_config(L.Params(nx=8, ny=8, nz=8), L.FullyPeriodicConfig())
    setattr(cfg, field, value)
    st, h = _create(cfg)
    assert st in (N.ERR_ARG, N.ERR_UNSUPPORTED) and not h.value


def test_null_arguments_are_errors_not_crashes():
    lib = N.lib()
    assert lib.lbman_create(None, None) == N.ERR_ARG
    assert lib.lbman_step(None, 1) == N.ERR_ARG
    assert lib.lbman_upload(None, None, None, None, None, None) == N.ERR_ARG
    assert lib.lbman_reduce(None, 1, None) == N.ERR_ARG
    assert lib.lbman_destroy(None) == N.OK


def test_presets_lower_to_faces():
    ch = [w.lower() for w in L.ChannelConfig().faces()]
    assert [f.ubc for f in ch] == [N.U_NOSLIP] * 4 + [N.U_PERIODIC] * 2
    sl = [w.lower() for w in L.SlitConfig().faces()]
    assert [f.ubc for f in sl] == [N.U_SPECULAR] * 2 + [N.U_PERIODIC] * 4
    lid = L.WallSpec(L.Anchoring(0.4, 1.0, 0.3), L.MovingWall(0.05, 0.0, 0.02)).lower()
    assert (lid.qbc, lid.s, lid.theta, lid.phi) == (N.Q_ANCHORING, 0.4, 1.0, 0.3)
    assert (lid.ubc, list(lid.uw)) == (N.U_MOVING, [0.05, 0.0, 0.02])
    assert L.periodicity_by_axis(L.ChannelConfig()) == [0, 0, 1]
    assert L.is_wall_by_face(L.SlitConfig()) == [True, True, False, False, False, False]
    assert L.PeriodicBC is L.FullyPeriodicConfig


def test_anchored_q_matches_oracle():
    from oracle import oracle as O
    a = L.Anchoring(0.3, 0.47, 0.33)
    f = O.Face()
    f.qbc, f.s, f.theta, f.phi = O.Q_ANCHORING, 0.3, 0.47, 0.33
    out = (C.c_double * 5)()
    O.lib().orc_anchored_q(C.byref(f), out)
    assert list(out) == list(L.boundary.anchored_q(a))
    # AnchoredQMagnitude (tests/unit/test_anchored_q.cc:18-30): HalfTrQ2 == S^2/3
    q = L.boundary.anchored_q(a)
    half = q[0] * q[0] + q[0] * q[3] + q[3] * q[3] + q[1] ** 2 + q[2] ** 2 + q[4] ** 2
    assert abs(half - 0.3 ** 2 / 3) < 1e-15


def test_host_fields_layout_roundtrip():
    p = L.Params(nx=3, ny=4, nz=5)
    g = L.LocalGrid.SingleRank(p)
    ff = L.FluidFields(g)
    ff.f[:] = np.arange(ff.f.size)
    soa = ff.f_soa()
    c, i = g.idx(2, 3, 4), 7
    assert soa[i * p.V + c] == ff.f[g.halo_idx(2, 3, 4, i)]
    ff2 = L.FluidFields(g)
    ff2.set_f_soa(soa)
    np.testing.assert_array_equal(ff2.f, ff.f)
    qf = L.QTensorFields(g)
    qf.set_q5(np.arange(5 * p.V, dtype=float))
    assert qf.qyy[0] == 3 * p.V
    qf.SwapWithNew()
    assert qf.qyy_new[0] == 3 * p.V
