"""Parity of the CUDA path (through the C ABI) with the reference.

* Golden fixtures (reference CPU solver outputs): the FP64 path must be
  bitwise equal, in both kernel organisations (split Q+force / LBM kernels
  and the fused one-kernel step).
* Larger seeded boxes against the CPU oracle: bitwise in FP64; FP32 and FP16
  deviation storage within stated relative max-norm bounds.
* The FP64 error gate: per-field max relative error max|a-b|/max|b| on rho,
  u and Q of at most 1e-12 after one step and 1e-9 after 100 steps (FP64).
"""
import numpy as np
import pytest

import lbman3d_b200 as L
from golden_util import load, names
from oracle import oracle as O

pytestmark = pytest.mark.gpu

KERNELS = [L._native.KERNELS_SPLIT, L._native.KERNELS_FUSED]


def relerr(a, b):
    d = np.max(np.abs(np.asarray(a) - np.asarray(b)))
    s = np.max(np.abs(b))
    return d / s if s > 0 else d


def sim_from(grid, faces, phys, upwind, precision=L.Precision.FP64, kernels=L._native.KERNELS_AUTO, tile=None):
    nx, ny, nz = grid
    p = L.Params(nx=nx, ny=ny, nz=nz, kQAdvection=L.Advection.Upwind if upwind else L.Advection.Centred, **phys)
    return L.Simulation(p, L.from_face_tuples(faces), precision, kernels, tile=tile)


@pytest.mark.parametrize("kernels", KERNELS, ids=["split", "fused"])
@pytest.mark.parametrize("name", names())
def test_fp64_matches_reference_bitwise(name, kernels):
    g = load(name)
    sim = sim_from(g["grid"], g["faces"], g["phys"], g["upwind"], kernels=kernels)
    sim.upload(g["in_rho"], g["in_u"], g["in_q"], None, g["in_force"])
    done = 0
    for k, t in enumerate(g["steps"]):
        for _ in range(t - done):
            if g["mode"] == "full":
                sim.step(1)
            elif g["mode"] == "q":
                sim.qtensor_step()
            else:
                sim.lbm_step()
        done = t
        out = sim.download(f=True, force=True)
        fields = {"full": ("rho", "u", "q", "f", "force"), "q": ("q",), "lbm": ("rho", "u", "f")}[g["mode"]]
        for f in fields:
            np.testing.assert_array_equal(out[f], g[f"s{k}_{f}"], err_msg=f"{name} step {t} {f}")


def _oracle_case(grid, faces, upwind=False, seed=3, **phys):
    nx, ny, nz = grid
    p = O.make_params(nx, ny, nz, faces, O.UPWIND if upwind else O.CENTRED, **phys)
    V = nx * ny * nz
    q = O.seeded_q(p, seed, O.equilibrium_order(p), 1e-3)
    rng = np.random.default_rng(seed)
    rho = 1.0 + 0.01 * rng.standard_normal(V)
    u = 0.005 * rng.standard_normal(3 * V)
    return p, rho, u, q


BIG = [
    ("periodic", (24, 20, 16), False),
    ("channel", (20, 26, 12), False),
    ("slit", (16, 33, 18), True),
    ("box_mixed", (13, 17, 19), False),
    ("lid", (31, 9, 14), True),
    ("qmixed", (15, 14, 13), True),
    ("qper_uwall", (18, 12, 10), False),
    ("walls", (34, 10, 9), False),
]


@pytest.mark.parametrize("kernels", KERNELS, ids=["split", "fused"])
@pytest.mark.parametrize("bc,grid,upwind", BIG)
def test_fp64_bitwise_vs_oracle_larger_boxes(bc, grid, upwind, kernels):
    from cases import BC
    p, rho, u, q = _oracle_case(grid, BC[bc], upwind, ALPHA=0.015, MU=0.002)
    ref = O.OracleSim(p)
    ref.set(rho, u, q)
    sim = sim_from(grid, BC[bc], dict(ALPHA=0.015, MU=0.002), upwind, kernels=kernels, tile=(14, 14, 5))
    sim.upload(rho, u, q)
    for n in (1, 7):
        ref.step(n)
        sim.step(n)
        a, b = sim.download(f=True), ref.get()
        for f in ("rho", "u", "q", "f"):
            np.testing.assert_array_equal(a[f], b[f], err_msg=f"{bc} {f}")


def test_fp64_error_gate_periodic_32():
    """FullyPeriodic 32^3, params.h defaults, seeded random director: <=1e-12
    after 1 step and <=1e-9 after 100 steps against the CPU oracle."""
    from cases import BC
    p, _, _, q = _oracle_case((32, 32, 32), BC["periodic"], seed=11)
    V = 32 ** 3
    rho, u = np.ones(V), np.zeros(3 * V)
    ref = O.OracleSim(p)
    ref.set(rho, u, q)
    sim = sim_from((32, 32, 32), BC["periodic"], {}, False)
    sim.upload(rho, u, q)
    ref.step(1)
    sim.step(1)
    a, b = sim.download(), ref.get()
    for f in ("rho", "u", "q"):
        assert relerr(a[f], b[f]) <= 1e-12, f
    ref.step(99)
    sim.step(99)
    a, b = sim.download(), ref.get()
    for f in ("rho", "u", "q"):
        assert relerr(a[f], b[f]) <= 1e-9, f


@pytest.mark.parametrize("precision,tol1,tol20", [(L.Precision.FP32, 1e-6, 2e-5), (L.Precision.FP16, 1e-3, 1e-2)],
                         ids=["fp32", "fp16"])
@pytest.mark.parametrize("bc", ["periodic", "channel", "slit", "box_mixed"])
def test_reduced_precision_vs_fp64_oracle(bc, precision, tol1, tol20):
    from cases import BC
    grid = (20, 18, 16)
    p, rho, u, q = _oracle_case(grid, BC[bc], ALPHA=0.01)
    ref = O.OracleSim(p)
    ref.set(rho, u, q)
    sim = sim_from(grid, BC[bc], dict(ALPHA=0.01), False, precision=precision)
    sim.upload(rho, u, q)
    ref.step(1)
    sim.step(1)
    a, b = sim.download(), ref.get()
    for f in ("rho", "u", "q"):
        e = relerr(a[f], b[f])
        assert e <= tol1, (f, e)
    ref.step(19)
    sim.step(19)
    a, b = sim.download(), ref.get()
    for f in ("rho", "u", "q"):
        e = relerr(a[f], b[f])
        assert e <= tol20, (f, e)


@pytest.mark.parametrize("precision", [L.Precision.FP64, L.Precision.FP32])
def test_reductions_match_oracle(precision):
    from cases import BC
    grid = (18, 14, 12)
    p, rho, u, q = _oracle_case(grid, BC["channel"], ALPHA=0.01)
    ref = O.OracleSim(p)
    ref.set(rho, u, q)
    ref.step(3)
    r = ref.get()
    sim = sim_from(grid, BC["channel"], dict(ALPHA=0.01), False, precision=precision)
    sim.upload(rho, u, q)
    sim.step(3)
    d = sim.reduce(L._native.DIAG_ALL)
    upast = np.zeros(3 * p.nx * p.ny * p.nz)
    lg = O.log_reduce(p, r["rho"], r["u"], upast)
    tol = 1e-12 if precision == L.Precision.FP64 else 2e-5
    V = p.nx * p.ny * p.nz
    absu = np.abs(r["u"]).reshape(3, V)
    # scale of each sum: the sum of the magnitudes of its terms
    scale = [V, *(r["rho"] * absu).sum(axis=1), lg[4], lg[5], lg[6], lg[7]]
    for k, key in enumerate(("mass", "px", "py", "pz", "kinetic_energy", "rel_change_num", "rel_change_den",
                             "umax2")):
        assert abs(d[key] - lg[k]) <= tol * scale[k] + 1e-18, key
    fe = O.free_energy(p, r["q"])
    assert abs(d["free_energy"] - fe) <= tol * abs(fe)
    S, dirs = O.order_director(p, r["q"])
    nflag = O.winding(p, dirs)[0]
    assert abs(d["defect_faces"] - nflag) <= (0 if precision == L.Precision.FP64 else 3)
    # relative-change numerator resets against the stored velocity
    d2 = sim.reduce(L._native.DIAG_FLOW)
    assert d2["rel_change_num"] == 0.0


def test_nan_is_reported_as_diverged():
    """A NaN planted in the host input propagates into the mass and the
    reduction returns the divergence status (SimIO::Log returning false)."""
    from cases import BC
    grid = (8, 8, 8)
    p, rho, u, q = _oracle_case(grid, BC["periodic"])
    rho = rho.copy()
    rho[17] = np.nan
    sim = sim_from(grid, BC["periodic"], {}, False)
    sim.upload(rho, u, q)
    sim.step(2)
    with pytest.raises(L._native.DivergedError):
        sim.reduce(L._native.DIAG_FLOW)
    d = sim.reduce(L._native.DIAG_FLOW, raise_on_nan=False)
    assert d["nan_detected"] == 1


def test_device_seeded_init_matches_host_generator():
    from cases import BC
    grid = (16, 12, 10)
    p = O.make_params(*grid, BC["periodic"])
    q_host = O.seeded_q(p, 5, 0.5, 1e-3)
    sim = sim_from(grid, BC["periodic"], {}, False)
    sim.init_seeded(5, 0.5, 1e-3)
    out = sim.download(f=True)
    np.testing.assert_allclose(out["q"], q_host, rtol=0, atol=1e-14)
    np.testing.assert_array_equal(out["rho"], np.ones(p.nx * p.ny * p.nz))


@pytest.mark.parametrize("bc,grid,upwind", BIG[:5], ids=[b[0] for b in BIG[:5]])
def test_in_place_streaming_across_organisation_switches(bc, grid, upwind):
    """The split organisations stream in place (one population buffer,
    AA pattern); the fused one keeps two buffers.  Switching between them
    mid-run converts the population layout: 3 in-place steps, 2 fused,
    3 in-place, with downloads of f after odd and even counts, must equal
    the CPU oracle bit for bit in FP64."""
    from cases import BC
    p, rho, u, q = _oracle_case(grid, BC[bc], upwind, ALPHA=0.015, MU=0.002)
    ref = O.OracleSim(p)
    ref.set(rho, u, q)
    sim = sim_from(grid, BC[bc], dict(ALPHA=0.015, MU=0.002), upwind, kernels=L._native.KERNELS_SPLIT,
                   tile=(14, 14, 5))
    sim.upload(rho, u, q)
    for n, kern in ((3, L._native.KERNELS_SPLIT), (2, L._native.KERNELS_FUSED), (1, L._native.KERNELS_SPLIT),
                    (2, L._native.KERNELS_SPLIT)):
        sim.set_shape(kern, 14, 14, 5)
        ref.step(n)
        sim.step(n)
        a, b = sim.download(f=True), ref.get()
        for f in ("rho", "u", "q", "f"):
            np.testing.assert_array_equal(a[f], b[f], err_msg=f"{bc} {f} after {kern}")
