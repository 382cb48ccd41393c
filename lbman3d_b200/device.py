"""GPU solver objects with the reference's interface, over the C ABI.

* :class:`DeviceFields` / :class:`DeviceSolver` mirror src/device_fields.h
  and src/device_solver.h: device-resident state, ``Initialize`` (upload),
  ``QTensorStep``, ``LBMStep``, ``CopyToHost``.
* :class:`LbmSolver` / :class:`QTensorSolver` mirror src/lbm_solver.h and
  src/qtensor_solver.h: they operate on host ``FluidFields`` /
  ``QTensorFields`` and run each call on the GPU (upload, step, download).
* :class:`Simulation` is a device-resident convenience handle used by the
  tests and the benchmark: arrays in, arrays out, ``step(n)``, ``reduce()``.

Every call goes to liblbman3d_b200.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N
from .boundary import BCConfig, SimBC
from .fields import FluidFields, LocalGrid, QTensorFields
from .params import Params, Precision


def InitializeComputeBackend(device: int = 0) -> str:
    """Device description (src/device_fields.h:21)."""
    buf = C.create_string_buffer(2048)
    N.check(N.lib().lbman_device_info(device, buf, len(buf)))
    return buf.value.decode()


def make_config(params: Params, bc: BCConfig, precision: int = Precision.FP64,
                kernels: int = N.KERNELS_AUTO, device: int = 0, tile=None) -> N.lbman_config:
    cfg = N.lbman_config()
    N.check(N.lib().lbman_config_init(C.byref(cfg)))
    cfg.nx, cfg.ny, cfg.nz = params.nx, params.ny, params.nz
    for k in ("DT", "kDensity", "TAUF", "L", "A", "B", "C", "LAMBDA", "GAMMA", "ALPHA", "MU"):
        setattr(cfg, k, float(getattr(params, k)))
    cfg.advection = int(params.kQAdvection)
    for i, w in enumerate(bc.faces()):
        cfg.face[i] = w.lower()
    cfg.precision = int(precision)
    cfg.kernels = int(kernels)
    cfg.device = int(device)
    if tile:
        cfg.tile_x, cfg.tile_y, cfg.zchunk, cfg.threads = (list(tile) + [0, 0, 0, 0])[:4]
    return cfg


class Simulation:
    """One device-resident box.  Host arrays follow the C ABI layout: u is 3
    blocks of V, q 5 blocks, f 15 direction-major blocks, all float64."""

    def __init__(self, params: Params, bc: BCConfig = None, precision: int = Precision.FP64,
                 kernels: int = N.KERNELS_AUTO, device: int = 0, tile=None):
        self.params = params
        self.bc = bc if bc is not None else SimBC()
        self.precision = precision
        self.cfg = make_config(params, self.bc, precision, kernels, device, tile)
        h = C.c_void_p()
        N.check(N.lib().lbman_create(C.byref(self.cfg), C.byref(h)))
        self._h = h

    @property
    def handle(self):
        return self._h

    @property
    def V(self):
        return self.params.V

    def close(self):
        if getattr(self, "_h", None):
            N.lib().lbman_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def upload(self, rho, u, q, f=None, force=None):
        c = lambda a: None if a is None else np.ascontiguousarray(a, dtype=np.float64)
        rho, u, q, f, force = c(rho), c(u), c(q), c(f), c(force)
        V = self.V
        for name, a, n in (("rho", rho, V), ("u", u, 3 * V), ("q", q, 5 * V), ("f", f, 15 * V),
                           ("force", force, 3 * V)):
            if a is not None and a.size != n:
                raise ValueError(f"{name} must have {n} values, got {a.size}")
        N.check(N.lib().lbman_upload(self._h, N.dptr(rho), N.dptr(u), N.dptr(q), N.dptr(f), N.dptr(force)))

    def init_seeded(self, seed: int, S0: float, sigma: float = 1e-3):
        N.check(N.lib().lbman_init_seeded(self._h, int(seed), float(S0), float(sigma)))

    def download(self, f=False, force=False):
        V = self.V
        out = dict(rho=np.empty(V), u=np.empty(3 * V), q=np.empty(5 * V))
        if f:
            out["f"] = np.empty(15 * V)
        if force:
            out["force"] = np.empty(3 * V)
        N.check(N.lib().lbman_download(self._h, N.dptr(out["rho"]), N.dptr(out["u"]), N.dptr(out["q"]),
                                       N.dptr(out.get("f")), N.dptr(out.get("force"))))
        return out

    def step(self, n: int = 1):
        N.check(N.lib().lbman_step(self._h, int(n)))

    def qtensor_step(self):
        N.check(N.lib().lbman_qtensor_step(self._h))

    def lbm_step(self):
        N.check(N.lib().lbman_lbm_step(self._h))

    def qtensor_setup(self):
        """Phase 1 of the Q stage: Q := Q_new, Sigma and tau kept on the
        device, body force := the Ericksen seed."""
        N.check(N.lib().lbman_qtensor_setup(self._h))

    def active_force(self):
        """Phase 2, the base activity model: force += -ALPHA div Q +
        div(Sigma + tau) - MU u."""
        N.check(N.lib().lbman_active_force(self._h))

    def download_stress(self):
        V = self.V
        sig, tau = np.empty(5 * V), np.empty(3 * V)
        N.check(N.lib().lbman_download_stress(self._h, N.dptr(sig), N.dptr(tau)))
        return sig, tau

    def upload_stress(self, sigma5, tau3):
        sig = np.ascontiguousarray(sigma5, dtype=np.float64)
        tau = np.ascontiguousarray(tau3, dtype=np.float64)
        if sig.size != 5 * self.V or tau.size != 3 * self.V:
            raise ValueError("sigma needs 5V values and tau 3V")
        N.check(N.lib().lbman_upload_stress(self._h, N.dptr(sig), N.dptr(tau)))

    def synchronize(self):
        N.check(N.lib().lbman_synchronize(self._h))

    def set_stream(self, stream_ptr: int):
        N.check(N.lib().lbman_set_stream(self._h, C.c_void_p(stream_ptr)))

    def reduce(self, flags: int = N.DIAG_ALL, raise_on_nan: bool = True):
        d = N.lbman_diag()
        st = N.lib().lbman_reduce(self._h, int(flags), C.byref(d))
        if st != N.OK and not (st == N.ERR_DIVERGED and not raise_on_nan):
            N.check(st)
        return {k: getattr(d, k) for k, _ in N.lbman_diag._fields_}

    def default_bins(self) -> int:
        """Shell count that covers every wavevector / separation of the box."""
        return int(max(self.params.nx, self.params.ny, self.params.nz) * 3 ** 0.5 / 2) + 2

    def velocity_spectrum(self, nbins: int = None):
        """Shell-averaged kinetic-energy spectrum E[b] and wavevectors per shell."""
        nb = int(nbins or self.default_bins())
        E, n = np.zeros(nb), np.zeros(nb)
        N.check(N.lib().lbman_velocity_spectrum(self._h, nb, N.dptr(E), N.dptr(n)))
        return E, n

    def q_correlation(self, nbins: int = None):
        """Radially averaged Q autocorrelation C[b], separations per shell and
        the 1/e correlation length (-1 if not reached)."""
        nb = int(nbins or self.default_bins())
        Cb, n, xi = np.zeros(nb), np.zeros(nb), C.c_double()
        N.check(N.lib().lbman_q_correlation(self._h, nb, N.dptr(Cb), N.dptr(n), C.byref(xi)))
        return Cb, n, xi.value

    def defect_lines(self, with_points: bool = True):
        """Disclination lines of the current Q, as the reference's
        DefectFinder: (info dict, points (n, 3) face centres, line offsets)."""
        info = N.lbman_defects()
        N.check(N.lib().lbman_defect_lines(self._h, C.byref(info), None, 0, None, 0))
        d = {k: getattr(info, k) for k, _ in N.lbman_defects._fields_}
        if not with_points:
            return d, None, None
        pts = np.zeros(3 * max(info.points, 1))
        off = np.zeros(info.lines + 1, dtype=np.int64)
        N.check(N.lib().lbman_defect_lines(self._h, C.byref(info), N.dptr(pts), pts.size,
                                           off.ctypes.data_as(C.POINTER(C.c_int64)), off.size))
        return d, pts[:3 * info.points].reshape(-1, 3), off

    def statistics(self) -> dict:
        """Mean and rms speed, defect plaquettes and their density per cell."""
        st = N.lbman_stats()
        N.check(N.lib().lbman_statistics(self._h, C.byref(st)))
        return {k: getattr(st, k) for k, _ in N.lbman_stats._fields_}

    def shape(self) -> dict:
        s = N.lbman_shape()
        N.check(N.lib().lbman_get_shape(self._h, C.byref(s)))
        return {k: getattr(s, k) for k, _ in N.lbman_shape._fields_}

    def set_shape(self, kernels: int, tile_x: int, tile_y: int, zchunk: int):
        s = N.lbman_shape(kernels, tile_x, tile_y, zchunk, 0, 0.0)
        N.check(N.lib().lbman_set_shape(self._h, C.byref(s)))

    def autotune(self, steps_per_trial: int = 5) -> dict:
        """Time every kernel organisation x tile x z-chunk candidate on the
        current state, keep the fastest, restore the state."""
        s, n = N.lbman_shape(), C.c_int()
        N.check(N.lib().lbman_autotune(self._h, int(steps_per_trial), C.byref(s), C.byref(n)))
        d = {k: getattr(s, k) for k, _ in N.lbman_shape._fields_}
        d["trials"] = n.value
        return d

    def launch_count(self) -> int:
        v = C.c_int64()
        N.check(N.lib().lbman_launch_count(self._h, C.byref(v)))
        return v.value

    def steps_done(self) -> int:
        v = C.c_int64()
        N.check(N.lib().lbman_steps_done(self._h, C.byref(v)))
        return v.value


class DeviceFields:
    """Device-resident fields (src/device_fields.h:23-56)."""

    def __init__(self, grid: LocalGrid, params: Params, bc: BCConfig = None,
                 precision: int = Precision.FP64, kernels: int = N.KERNELS_AUTO, device: int = 0):
        self.grid = grid
        self.sim = Simulation(params, bc, precision, kernels, device)

    def Initialize(self, ff: FluidFields, qf: QTensorFields):
        """Upload populations, body force, density, velocity and Q
        (src/cuda/device_fields.cu:79-115; the AoS->SoA transpose of f is done
        here as there).  Unlike the reference, rho and u are uploaded too, so
        the first Q step sees the host velocity as the CPU path does."""
        self.sim.upload(ff.rho, ff.u3(), qf.q5(), ff.f_soa(), ff.force3())

    def CopyToHost(self, ff: FluidFields, qf: QTensorFields):
        """rho, u and Q back to the host (src/cuda/device_fields.cu:118-127)."""
        out = self.sim.download()
        V = self.grid.Volume()
        ff.rho[:] = out["rho"]
        ff.ux[:], ff.uy[:], ff.uz[:] = out["u"][:V], out["u"][V:2 * V], out["u"][2 * V:]
        qf.set_q5(out["q"])


class DeviceSolver:
    """DeviceSolver<BC> (src/device_solver.h:10-17).  The BC lives in the
    DeviceFields' configuration, so the solver itself is stateless."""

    def __init__(self, bc: BCConfig = None):
        self.bc = bc

    def Initialize(self, df: DeviceFields):
        pass  # lattice tables are compile-time constants of the kernels

    def QTensorStep(self, df: DeviceFields):
        df.sim.qtensor_step()

    def LBMStep(self, df: DeviceFields):
        df.sim.lbm_step()

    def Step(self, df: DeviceFields):
        df.sim.step(1)


class LbmSolver:
    """LbmSolver<BC> on host fields (src/lbm_solver.h:12-21), each call run on
    the GPU: upload, step, download."""

    def __init__(self, bc: BCConfig, params: Params, precision: int = Precision.FP64, device: int = 0):
        self.bc, self.params = bc, params
        self.sim = Simulation(params, bc, precision, N.KERNELS_SPLIT, device)

    def Initialize(self, ff: FluidFields):
        """f = f_eq(rho, u) (src/lbm_solver.tpp:35-62)."""
        V = self.params.V
        self.sim.upload(ff.rho, ff.u3(), np.zeros(5 * V))
        ff.set_f_soa(self.sim.download(f=True)["f"])

    def LatticeBoltzmannStep(self, ff: FluidFields):
        V = self.params.V
        self.sim.upload(ff.rho, ff.u3(), np.zeros(5 * V), ff.f_soa(), ff.force3())
        self.sim.lbm_step()
        out = self.sim.download(f=True)
        ff.set_f_soa(out["f"])
        ff.rho[:] = out["rho"]
        ff.ux[:], ff.uy[:], ff.uz[:] = out["u"][:V], out["u"][V:2 * V], out["u"][2 * V:]


class QTensorSolver:
    """QTensorSolver<BC> on host fields (src/qtensor_solver.h:23-52), run on
    the GPU with the reference's two-phase contract:
    StepAndSetupBodyForce writes Q_new (Q and Q_new exchanged as SwapWithNew
    leaves them), Sigma, tau and the Ericksen seed of the body force; the
    overridable SetActiveStressAndComputeBodyForce adds the active, passive
    and friction terms, and a subclass override replaces it
    (src/qtensor_solver.h:11-21).  Step runs both phases; an object of
    exactly this class (nothing overridden) takes one fused GPU pass, which
    leaves qf.Sigma_* / qf.Tau_* as they were."""

    SIGMA = ("Sigma_xx", "Sigma_xy", "Sigma_xz", "Sigma_yy", "Sigma_yz")
    TAU = ("Tau_xy", "Tau_xz", "Tau_yz")

    def __init__(self, bc: BCConfig, params: Params, precision: int = Precision.FP64, device: int = 0):
        self.bc, self.params = bc, params
        self.sim = Simulation(params, bc, precision, N.KERNELS_SPLIT, device)

    def Initialize(self, qf: QTensorFields, seed: int = 0):
        """Uniform director along z at S_eq plus uniform noise of amplitude NOISE
        (src/qtensor_solver.tpp:14-48), seeded here for reproducibility."""
        from .params import EquilibriumScalarOrder
        rng = np.random.default_rng(seed)
        s_eq = EquilibriumScalarOrder(self.params)
        V, nz = self.params.V, self.params.NOISE
        qf.qxx[:] = -s_eq / 3.0 + rng.uniform(-nz, nz, V)
        qf.qxy[:] = rng.uniform(-nz, nz, V)
        qf.qxz[:] = rng.uniform(-nz, nz, V)
        qf.qyy[:] = -s_eq / 3.0 + rng.uniform(-nz, nz, V)
        qf.qyz[:] = rng.uniform(-nz, nz, V)

    def _store(self, qf: QTensorFields, ff: FluidFields, out):
        V = self.params.V
        for k, c in enumerate(qf.COMPS):
            getattr(qf, c + "_new")[:] = getattr(qf, c)
            getattr(qf, c)[:] = out["q"][k * V:(k + 1) * V]
        F = out["force"]
        ff.fx[:], ff.fy[:], ff.fz[:] = F[:V], F[V:2 * V], F[2 * V:]

    def StepAndSetupBodyForce(self, qf: QTensorFields, ff: FluidFields):
        """Phase 1 (src/qtensor_solver.tpp:51-147) on the GPU."""
        V = self.params.V
        self.sim.upload(ff.rho, ff.u3(), qf.q5())
        self.sim.qtensor_setup()
        self._store(qf, ff, self.sim.download(force=True))
        sig, tau = self.sim.download_stress()
        for k, c in enumerate(self.SIGMA):
            getattr(qf, c)[:] = sig[k * V:(k + 1) * V]
        for k, c in enumerate(self.TAU):
            getattr(qf, c)[:] = tau[k * V:(k + 1) * V]

    def SetActiveStressAndComputeBodyForce(self, ff: FluidFields, qf: QTensorFields):
        """Phase 2, the base activity model (src/qtensor_solver.tpp:155-217),
        on the GPU; override to change the activity model."""
        V = self.params.V
        self.sim.upload(ff.rho, ff.u3(), qf.q5(), force=ff.force3())
        self.sim.upload_stress(np.concatenate([getattr(qf, c) for c in self.SIGMA]),
                               np.concatenate([getattr(qf, c) for c in self.TAU]))
        self.sim.active_force()
        F = self.sim.download(force=True)["force"]
        ff.fx[:], ff.fy[:], ff.fz[:] = F[:V], F[V:2 * V], F[2 * V:]

    def Step(self, qf: QTensorFields, ff: FluidFields):
        if type(self) is QTensorSolver:
            self.sim.upload(ff.rho, ff.u3(), qf.q5())
            self.sim.qtensor_step()
            self._store(qf, ff, self.sim.download(force=True))
            return
        self.StepAndSetupBodyForce(qf, ff)
        self.SetActiveStressAndComputeBodyForce(ff, qf)
