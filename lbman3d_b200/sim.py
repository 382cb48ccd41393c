"""Simulation driver over the GPU solver: the reference's ActiveNematicSim
(src/active_nematic.h:34-142), its lbm.log output (src/sim_io.cc:32-166),
frame export and the main / benchmark loops (src/main.cc, src/benchmark.cc).

    python -m lbman3d_b200.sim --nx 20 --ny 100 --nz 100 --bc slit_noslip \\
        --steps 10000 --save-interval 100 [--export data]
    python -m lbman3d_b200.sim --benchmark

Log lines keep the reference's wording and number format (C++ std::format
defaults, restated by ``cxx_format``) so tools that parse lbm.log -- the
reference's monitor.py among them -- read them unchanged.  Frames: the
reference writes VTKHDF through HDF5, which this library does not link; each
frame is instead one raw little-endian file (``frame_{k:06d}.bin``) with a
JSON header beside it listing the arrays, their dtype, shape ([nz, ny, nx]
point data, the VTKHDF ordering) and byte offset: rho, velocity (3),
Q (xx, xy, xz, yy, yz), the scalar order S and the director (3), plus the
disclination polylines (points xyz, line offsets) of the same step.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import sys

import numpy as np

from . import _native as N
from .boundary import ChannelConfig, FullyPeriodicConfig, SlitConfig, SlitNoSlipConfig
from .device import Simulation, InitializeComputeBackend
from .params import EquilibriumScalarOrder, Params, Precision


def cxx_format(x) -> str:
    """std::format("{}", x): integers as-is; doubles in the shortest form that
    reads back exactly, fixed or scientific (%e-style exponent of at least
    two digits), whichever is shorter, fixed on a tie."""
    if isinstance(x, (bool, np.bool_)):
        return "true" if x else "false"
    if isinstance(x, (int, np.integer)):
        return str(int(x))
    x = float(x)
    if math.isnan(x):
        return "-nan" if math.copysign(1.0, x) < 0 else "nan"
    if math.isinf(x):
        return "-inf" if x < 0 else "inf"
    sign = "-" if math.copysign(1.0, x) < 0 else ""
    a = abs(x)
    if a == 0.0:
        return sign + "0"
    s = repr(a)
    m, e = (s.split("e") + ["0"])[:2] if "e" in s else (s, "0")
    ip, fp = (m.split(".") + [""])[:2] if "." in m else (m, "")
    digits = (ip + fp).lstrip("0")
    exp10 = int(e) - len(fp)
    stripped = digits.rstrip("0")
    exp10 += len(digits) - len(stripped)
    digits = stripped or "0"
    n = len(digits)
    sci_exp = n - 1 + exp10
    sci = digits[0] + ("." + digits[1:] if n > 1 else "") + "e" + ("-" if sci_exp < 0 else "+") + \
        f"{abs(sci_exp):02d}"
    if exp10 >= 0:
        fixed = digits + "0" * exp10
    else:
        p = n + exp10
        fixed = digits[:p] + "." + digits[p:] if p > 0 else "0." + "0" * (-p) + digits
    return sign + (fixed if len(fixed) <= len(sci) else sci)


BCS = {"periodic": FullyPeriodicConfig, "channel": ChannelConfig, "slit": SlitConfig,
       "slit_noslip": SlitNoSlipConfig}


class ActiveNematicSim:
    """ActiveNematicSim<BC> on the GPU solver.  The initial state is the
    reference's (director along z at S_eq plus U(-NOISE, NOISE) noise, f =
    f_eq at rho = kDensity, u = 0; src/qtensor_solver.tpp:14-48) drawn from a
    seeded generator, or the benchmark workloads' seeded random director
    with ``init="random_director"``."""

    def __init__(self, params: Params, bc=None, precision: int = Precision.FP64, log_path: str = "lbm.log",
                 seed: int = 0, init: str = "reference", bc_name: str = None, device: int = 0):
        self.p = params
        self.bc = bc if bc is not None else SlitNoSlipConfig()
        self.sim = Simulation(params, self.bc, precision, device=device)
        self.time_step = 0
        self.num_files_exported = 0
        self._log = open(log_path, "w") if log_path else None
        V = params.V
        if init == "random_director":
            self.sim.init_seeded(seed, EquilibriumScalarOrder(params), 1e-3)
        else:
            r = np.random.default_rng(seed)
            s_eq = EquilibriumScalarOrder(params)
            q = np.empty((5, V))
            noise = lambda: r.uniform(-params.NOISE, params.NOISE, V)
            q[0] = -s_eq / 3.0 + noise()
            q[1] = noise()
            q[2] = noise()
            q[3] = -s_eq / 3.0 + noise()
            q[4] = noise()
            self.sim.upload(np.full(V, params.kDensity), np.zeros(3 * V), q.ravel())
        self.LogSetupSummary(bc_name or type(self.bc).__name__, InitializeComputeBackend(device))

    # --- stepping (src/active_nematic.h:84-108) ---------------------------------
    def QTensorStep(self):
        self.sim.qtensor_step()

    def LBMStep(self):
        self.sim.lbm_step()

    def Step(self):
        self.sim.step(1)
        self.time_step += 1

    def GetTimeStep(self) -> int:
        return self.time_step

    # --- log (src/sim_io.cc:32-166) ------------------------------------------------
    def _println(self, s=""):
        if self._log:
            self._log.write(s + "\n")

    def LogSetupSummary(self, bc_name: str, backend_info: str):
        p, f = self.p, cxx_format
        out = ["Hybrid Lattice Boltzmann simulation for 3D active nematics\n",
               "##########################################################",
               "#####################   Parameters   #####################",
               "##########################################################", "",
               "--- Compute backend ---", f"  {backend_info}", "",
               "--- Grid ---", f"  nx = {p.nx}, ny = {p.ny}, nz = {p.nz}", f"  DX = {f(1.0)}, DY = {f(1.0)}, DZ = {f(1.0)}",
               f"  BC = {bc_name}", "",
               "--- Time ---", f"  DT (numerical)      = {f(p.DT)}", "",
               "--- LBM ---", f"  TAUF                = {f(p.TAUF)}",
               f"  Kinematic Viscosity = {f(p.kinematicViscosity)}", f"  omega               = {f(p.omega)}",
               f"  omega_prime         = {f(p.omega_prime)}", f"  omega_forcing       = {f(p.omega_forcing)}", "",
               "--- Free energy ---", f"  L (Frank elasticity) = {f(p.L)}", f"  A                    = {f(p.A)}",
               f"  B                    = {f(p.B)}", f"  C                    = {f(p.C)}", "",
               "--- Q-tensor dynamics ---", f"  GAMMA (rot. viscosity^-1) = {f(p.GAMMA)}",
               f"  LAMBDA (flow-aligning)    = {f(p.LAMBDA)}", f"  NOISE                     = {f(p.NOISE)}", "",
               "--- Activity & friction ---", f"  ALPHA (numerical)  = {f(p.ALPHA)}",
               f"  MU (linear friction) = {f(p.MU)}", "",
               "##########################################################"]
        for line in out:
            self._println(line)

    def Log(self, track_nematic_energy: bool = False) -> bool:
        """One lbm.log line (SimIO::Log); False when mass or momentum is NaN."""
        flags = N.DIAG_FLOW | (N.DIAG_ENERGY if track_nematic_energy else 0)
        d = self.sim.reduce(flags, raise_on_nan=False)
        ndisc = -1
        if min(self.p.nx, self.p.ny, self.p.nz) >= 2 and not d["nan_detected"]:
            ndisc = self.sim.defect_lines(with_points=False)[0]["lines"]
        ke = d["kinetic_energy"]
        te = ke + (d["free_energy"] if track_nematic_energy else 0.0)
        f = cxx_format
        num, den = d["rel_change_num"], d["rel_change_den"]
        if den != 0:
            rel = num / den
        else:  # IEEE division as the reference does it (0/0 is the x86 default NaN, sign bit set)
            rel = math.copysign(math.inf, num) if num != 0 else math.copysign(math.nan, -1.0)
        self._println(f"Time {self.time_step}: Mass: {f(d['mass'])}, Px: {f(d['px'])}, Py: {f(d['py'])}, "
                      f"Pz: {f(d['pz'])}, Kinetic Energy: {f(ke)}, Total Energy: {f(te)}, Relative Error: {f(rel)}, "
                      f"NumDisclinations: {ndisc}, Nematic Energy: {f(te - ke)}, Max |u|: {f(math.sqrt(d['umax2']))}")
        if self._log:
            self._log.flush()
        if d["nan_detected"]:
            self._println(f"DIVERGED at time step {self.time_step} — aborting.")
            return False
        return True

    # --- frames ----------------------------------------------------------------------
    def Export(self, path: str):
        os.makedirs(path, exist_ok=True)
        p = self.p
        out = self.sim.download()
        V = p.V
        shape = [p.nz, p.ny, p.nx]
        q = out["q"].reshape(5, V)
        S, director = _order_director(q)
        info, pts, off = self.sim.defect_lines() if min(p.nx, p.ny, p.nz) >= 2 else ({}, np.zeros((0, 3)),
                                                                                      np.zeros(1, np.int64))
        arrays = [("rho", out["rho"].reshape(shape)), ("velocity", out["u"].reshape(3, *shape)),
                  ("Q", q.reshape(5, *shape)), ("S", S.reshape(shape)), ("director", director.reshape(3, *shape)),
                  ("disclination_points", pts), ("disclination_offsets", off)]
        k = self.num_files_exported
        header = {"step": self.time_step, "grid": [p.nx, p.ny, p.nz], "arrays": []}
        with open(os.path.join(path, f"frame_{k:06d}.bin"), "wb") as fh:
            offset = 0
            for name, a in arrays:
                a = np.ascontiguousarray(a)
                header["arrays"].append({"name": name, "dtype": str(a.dtype), "shape": list(a.shape),
                                         "offset": offset})
                fh.write(a.tobytes())
                offset += a.nbytes
        with open(os.path.join(path, f"frame_{k:06d}.json"), "w") as fh:
            json.dump(header, fh, indent=1)
        self.num_files_exported += 1

    def close(self):
        if self._log:
            self._println("LBM program exited.")
            self._log.close()
            self._log = None
        self.sim.close()


def _order_director(q):
    """Largest eigenvalue and its eigenvector per cell (QtensorToOrderDirector
    semantics, src/analysis_fields.cc:59-93, by a symmetric eigensolver)."""
    xx, xy, xz, yy, yz = q
    M = np.empty((q.shape[1], 3, 3))
    M[:, 0, 0], M[:, 0, 1], M[:, 0, 2] = xx, xy, xz
    M[:, 1, 0], M[:, 1, 1], M[:, 1, 2] = xy, yy, yz
    M[:, 2, 0], M[:, 2, 1], M[:, 2, 2] = xz, yz, -(xx + yy)
    w, v = np.linalg.eigh(M)
    return w[:, -1], np.ascontiguousarray(v[:, :, -1].T)


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="ActiveNematicSim on the B200 solver (reference main / benchmark)")
    ap.add_argument("--nx", type=int, default=20)
    ap.add_argument("--ny", type=int, default=100)
    ap.add_argument("--nz", type=int, default=100)
    ap.add_argument("--bc", choices=sorted(BCS), default="slit_noslip")
    ap.add_argument("--alpha", type=float, default=None)
    ap.add_argument("--precision", choices=["fp64", "fp32", "fp16"], default="fp64")
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--save-interval", type=int, default=100)
    ap.add_argument("--export", default=None, help="frame directory (reference: data)")
    ap.add_argument("--log", default="lbm.log")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--benchmark", action="store_true", help="the reference benchmark.cc loop and report")
    a = ap.parse_args(argv)
    kw = dict(nx=a.nx, ny=a.ny, nz=a.nz)
    if a.alpha is not None:
        kw["ALPHA"] = a.alpha
    p = Params(**kw)
    prec = {"fp64": Precision.FP64, "fp32": Precision.FP32, "fp16": Precision.FP16}[a.precision]
    sim = ActiveNematicSim(p, BCS[a.bc](), prec, a.log, a.seed, bc_name=a.bc)
    try:
        if a.benchmark:
            return _benchmark(sim)
        for t in range(a.steps):
            if t % a.save_interval == 0:
                print(f"Step {t}")
                if a.export:
                    sim.Export(a.export)
                if not sim.Log():
                    print(f"Simulation diverged at step {t} — exiting.", file=sys.stderr)
                    return 1
            sim.Step()
        return 0
    finally:
        sim.close()


def _benchmark(sim: ActiveNematicSim, warmup: int = 10, steps: int = 1000) -> int:
    import torch
    print(f"Running on: {InitializeComputeBackend()}")
    for _ in range(warmup):
        sim.Step()
    st = torch.cuda.current_stream()
    sim.sim.set_stream(st.cuda_stream)
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    ms_q = ms_l = 0.0
    for _ in range(steps):
        e[0].record(st)
        sim.QTensorStep()
        e[1].record(st)
        sim.LBMStep()
        e[2].record(st)
        e[2].synchronize()
        ms_q += e[0].elapsed_time(e[1])
        ms_l += e[1].elapsed_time(e[2])
    tot = ms_q + ms_l
    p = sim.p
    print(f"NX={p.nx} NY={p.ny} NZ={p.nz}\nSteps(successful): {steps}({steps})\n"
          f"  QTensor : {ms_q / steps:.3f} ms/step ({100 * ms_q / tot:.1f}%)\n"
          f"  LBM     : {ms_l / steps:.3f} ms/step ({100 * ms_l / tot:.1f}%)\n"
          f"  Total   : {tot / steps:.3f} ms/step\n"
          f"  MLUPS   : {p.V * steps / (tot * 1e3):.1f}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
