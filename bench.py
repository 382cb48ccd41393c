"""Benchmark of the sm_100a time step (contract: one JSON line on rank 0).

Default workload: FullyPeriodicConfig 512x512x512, params.h defaults with
zeta (ALPHA) = 0.01 and LAMBDA = 0.3, centred advection, FP32 compute with
populations stored as FP32 deviations, seeded random-director initial
condition (the precision configuration, the largest single-GPU one).  A
"step" is one full time step (Q-tensor update + body force + D3Q15
collide/stream) over the whole box.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload periodic512|slit64|channel20|periodic32]
                    [--precision fp32|fp64|fp16]

value    : MLUPS (million lattice-cell updates per second), all GPUs, device
           resident fields, timed with CUDA events on the solver's stream,
           max over ranks.
e2e      : the same metric through the C ABI with host (pinned) buffers: each
           e2e step uploads rho/u/Q, runs kSaveInterval = 100 solver steps and
           downloads rho/u/Q, as ActiveNematicSim's save cycle does.
roofline : algorithmic bytes per cell update of the dominant kernel (Q+force:
           Q, u read, Q_new, F written; LBM: f*, F read, f*, u written) x cells
           / its average duration, against the measured HBM copy bandwidth;
           the whole step against 184 B/cell (f 15+15, Q 5+5, u 3+3 words).
error_vs_fp64 : FP32 and FP16-storage fields against the FP64 path (bitwise
           the reference's arithmetic) from the same seed after 2000 steps.
--impl reference : the reference's own OpenMP CPU solver (oracle/_ref build
           of its sources) on this machine's host cores, bounded sample.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: (nx, ny, nz, bc, ALPHA, ref_build)
    "periodic512": (512, 512, 512, "periodic", 0.01, "b_p512"),
    "slit64": (64, 256, 256, "slit", 0.01, "b_slit"),
    "channel20": (20, 100, 100, "channel", 0.01, "b_channel"),
    "periodic32": (32, 32, 32, "periodic", 0.023, "b_p32"),
    # a 512^2 x 64 slab of the precision configuration: profiler captures
    # (a few GB on the device), scaled per cell to the full box
    "periodic512x64": (512, 512, 64, "periodic", 0.01, None),
    # the largest FP32 box one GPU holds (159 GB); run with --no-extras and a
    # pinned --kernels/--tile (the autotuner's state snapshot does not fit)
    "periodic1024": (1024, 1024, 1024, "periodic", 0.01, None),
}
SEED, S0, SIGMA = 1234, 0.5, 1e-3
# Host bytes per cell of the reference's CPU solver: FluidFields (f, f_new,
# force, rho, u: 37 doubles) + QTensorFields (Q, Q_new, Sigma, tau: 18) and the
# seeded field while it is injected (5).
REF_HOST_BYTES_PER_CELL = 8 * (37 + 18 + 5)
BYTES_PER_CELL = {"fp64": 368, "fp32": 184, "fp16": 124}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(workload, precision, kernel):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, or None."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_{workload}_{precision}.md")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.strip().startswith("traffic_bytes_per_launch:"):
            try:
                return float(line.split(":", 1)[1].strip())
            except ValueError:
                return None
    return None


def bc_for(name):
    import lbman3d_b200 as L
    return {"slit": L.SlitConfig, "channel": L.ChannelConfig, "periodic": L.FullyPeriodicConfig}[name]()


class ClockSampler:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device, self.proc, self.out = device, None, None

    def __enter__(self):
        try:
            self.out = tempfile.TemporaryFile(mode="w+")
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.device)], stdout=self.out,
                                         stderr=subprocess.DEVNULL)
            time.sleep(0.3)
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc:
            time.sleep(0.2)
            self.proc.terminate()
            self.proc.wait(timeout=10)

    def summary(self):
        if not self.proc:
            return None
        self.out.seek(0)
        rows = [r.split(",") for r in self.out.read().strip().splitlines() if r.count(",") >= 7]
        if not rows:
            return None
        sm = [float(r[0]) for r in rows if r[0].strip().replace(".", "").isdigit()]
        mx = max(float(r[1]) for r in rows)
        reasons = set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            for nm, v in zip(names, r[4:8]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(rows)}


def make_sim(workload, precision, device, kernels="auto", tile=None):
    import lbman3d_b200 as L
    nx, ny, nz, bc, alpha, _ = WORKLOADS[workload]
    p = L.Params(nx=nx, ny=ny, nz=nz, ALPHA=alpha)
    prec = {"fp64": L.Precision.FP64, "fp32": L.Precision.FP32, "fp16": L.Precision.FP16}[precision]
    kern = {"auto": L._native.KERNELS_AUTO, "split": L._native.KERNELS_SPLIT, "fused": L._native.KERNELS_FUSED,
            "pair": L._native.KERNELS_SPLIT_PAIR}[kernels]
    sim = L.Simulation(p, bc_for(bc), prec, kern, device=device, tile=tile)
    return sim, p


def time_device(sim, steps, warmup, stream):
    """Device-resident steps timed with CUDA events on the solver's stream."""
    import torch
    sim.init_seeded(SEED, S0, SIGMA)
    sim.step(warmup)
    sim.synchronize()
    l0 = sim.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    sim.step(steps)
    e1.record(stream)
    e1.synchronize()
    return e0.elapsed_time(e1), sim.launch_count() - l0


def kernel_breakdown(sim, kernels, precision, V, stream, n):
    """Average duration of each kernel of the step, CUDA events around each
    launch on the solver's stream, with the algorithmic bytes per cell each
    one must move (state words read + written, body force included)."""
    import torch
    rb = 8 if precision == "fp64" else 4
    sb = {"fp64": 8, "fp32": 4, "fp16": 2}[precision]
    if kernels == "fused":
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        sim.step(2)
        e0.record(stream)
        sim.step(n)
        e1.record(stream)
        e1.synchronize()
        return {"fused_step": {"ms": e0.elapsed_time(e1) / n, "bytes_per_cell": 30 * sb + 16 * rb}}
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(n)]
    sim.step(2)
    for a, b, c in ev:
        a.record(stream)
        sim.qtensor_step()
        b.record(stream)
        sim.lbm_step()
        c.record(stream)
    ev[-1][2].synchronize()
    tq = sum(a.elapsed_time(b) for a, b, _ in ev) / n
    tl = sum(b.elapsed_time(c) for _, b, c in ev) / n
    # Q+force: Q, u read; Q_new, F written.  LBM: f*, F read; f*, u written.
    return {"qforce": {"ms": tq, "bytes_per_cell": 16 * rb}, "lbm": {"ms": tl, "bytes_per_cell": 30 * sb + 6 * rb}}


def ensemble_vs_sequential(device, stream, nboxes=96, steps=200, seq_steps=40):
    """Batching workload: 96 seeded boxes (sides in {24..96}, half periodic,
    half slit, zeta log-uniform in [1e-3, 3e-2], LAMBDA uniform in
    [0.1, 0.7]), FP32, advanced together by the ensemble runner (autotuned,
    CUDA-graph replay) versus the same boxes run one after another through
    the single-box solver (each autotuned).  Aggregate MLUPS both ways."""
    import torch
    import lbman3d_b200 as L
    boxes = L.draw_boxes(nboxes, seed=2024)
    cells = sum(p.V for p, _ in boxes)
    ens = L.Ensemble(boxes, L.Precision.FP32, device=device)
    ens.set_stream(stream.cuda_stream)
    ens.init_seeded(7)
    tuned = ens.autotune(steps_per_trial=3)
    ens.step(5)
    ens.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    l0 = ens.info()["launches"]
    e0.record(stream)
    ens.step(steps)
    e1.record(stream)
    e1.synchronize()
    t_ens = e0.elapsed_time(e1)
    launches = ens.info()["launches"] - l0
    ens.close()
    t_seq = 0.0
    for i, (p, bc) in enumerate(boxes):
        s = L.Simulation(p, bc, L.Precision.FP32, device=device)
        s.set_stream(stream.cuda_stream)
        s.init_seeded(7 + i, 0.5, 1e-3)
        s.autotune(steps_per_trial=2)
        s.step(3)
        s.synchronize()
        e0.record(stream)
        s.step(seq_steps)
        e1.record(stream)
        e1.synchronize()
        t_seq += e0.elapsed_time(e1)
        s.close()
    m_ens = cells * steps / (t_ens * 1e3)
    m_seq = cells * seq_steps / (t_seq * 1e3)
    return {"boxes": nboxes, "cells": cells, "ensemble_mlups": m_ens, "sequential_mlups": m_seq,
            "speedup": m_ens / m_seq, "ensemble_steps": steps, "sequential_steps_per_box": seq_steps,
            "ensemble_launches_per_step": launches / steps,
            "shape": {k: tuned[k] for k in ("kernels", "tile_x", "tile_y", "zchunk")}}


def max_rel_err(a, b, chunk=1 << 24):
    """max|a - b| / max|b| over one field, in chunks (bounded temporaries)."""
    num = den = 0.0
    for i in range(0, a.size, chunk):
        x, y = a[i:i + chunk], b[i:i + chunk]
        num = max(num, float(np.max(np.abs(x - y))))
        den = max(den, float(np.max(np.abs(y))))
    return num / max(den, 1e-300)


def errors_vs_fp64(workload, precisions, device, nsteps):
    """Per-field max relative error of each precision against the FP64 path
    (bitwise the reference arithmetic) on the same seed after nsteps; one FP64
    run serves every precision.  Device time of each run is reported too."""
    import torch

    def run(prec):
        s, _ = make_sim(workload, prec, device)
        s.init_seeded(SEED, S0, SIGMA)
        s.synchronize()
        t0 = time.perf_counter()
        s.step(nsteps)
        s.synchronize()
        dt = time.perf_counter() - t0
        out = s.download()
        s.close()
        torch.cuda.empty_cache()
        return out, dt

    ref, t_ref = run("fp64")
    res = {"steps": nsteps, "fp64_run_s": t_ref,
           "metric": "max|a-b|/max|b| per field against the FP64 path (bitwise the reference arithmetic), "
                     "same seed, same steps"}
    for prec in precisions:
        x, dt = run(prec)
        res[prec] = {f: max_rel_err(x[f], ref[f]) for f in ("rho", "u", "q")}
        res[prec]["run_s"] = dt
        res[prec]["nan"] = bool(not all(np.isfinite(x[f]).all() for f in ("rho", "u", "q")))
        del x
    return res


def host_mem_available():
    """MemAvailable of this host in bytes (None where /proc/meminfo is absent)."""
    try:
        with open("/proc/meminfo") as fh:
            for line in fh:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) * 1024
    except OSError:
        pass
    return None


def reduce_max(value, world, device):
    """The maximum of a per-rank float over all ranks (the value itself on one
    rank).  Every rank must call it, in the same order."""
    if world == 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(cells_per_rank, steps, world, ms_max):
    """MLUPS of the whole job: every rank advanced its own box of
    cells_per_rank cells by `steps` steps, the slowest rank in ms_max."""
    return world * cells_per_rank * steps / (ms_max * 1e3)


def time_e2e(sim, p, iters, stream, save_interval=100, world=1, device=None):
    import torch
    V = p.V
    pin = lambda n: torch.empty(n, dtype=torch.float64, pin_memory=True).numpy()
    rho, u, q = pin(V), pin(3 * V), pin(5 * V)
    orho, ou, oq = pin(V), pin(3 * V), pin(5 * V)
    from lbman3d_b200 import _native as N
    lib, h = N.lib(), sim.handle
    sim.init_seeded(99, S0, SIGMA)
    N.check(lib.lbman_download(h, N.dptr(rho), N.dptr(u), N.dptr(q), None, None))

    def cycle():
        N.check(lib.lbman_upload(h, N.dptr(rho), N.dptr(u), N.dptr(q), None, None))
        N.check(lib.lbman_step(h, save_interval))
        N.check(lib.lbman_download(h, N.dptr(orho), N.dptr(ou), N.dptr(oq), None, None))

    cycle()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(iters):
        cycle()
    e1.record(stream)
    e1.synchronize()
    ms = reduce_max(e0.elapsed_time(e1), world, device)
    mlups = whole_job_rate(V, save_interval * iters, world, ms)
    return {"value": mlups, "unit": "MLUPS", "h2d_bytes_per_step": world * 9 * V * 8,
            "d2h_bytes_per_step": world * 9 * V * 8, "solver_steps_per_step": save_interval, "steps": iters}


def reference_cpu(workload, max_steps, warmup):
    """The reference's OpenMP CPU solver on the host cores (oracle/_ref build
    of its own sources), on the seeded initial condition of the workload,
    generated inside the driver.  Raises RuntimeError when the host cannot
    hold the reference's fields."""
    from oracle import build_ref
    nx, ny, nz, bc, alpha, tag = WORKLOADS[workload]
    exe = build_ref.driver_path(tag) if tag else None
    cores = os.cpu_count() or 1
    V = nx * ny * nz
    need = REF_HOST_BYTES_PER_CELL * V
    avail = host_mem_available()
    if avail is not None and need > 0.9 * avail:
        raise RuntimeError(f"the reference CPU solver needs {need / 1e9:.0f} GB of host memory for "
                           f"{nx}x{ny}x{nz}; {avail / 1e9:.0f} GB available")
    if exe and os.path.exists(exe):
        r = subprocess.run([exe, "--bench", bc, str(SEED), repr(S0), repr(SIGMA), str(warmup), str(max_steps)],
                           capture_output=True, text=True,
                           env=dict(os.environ, LBMAN_REF_THREADS=str(cores), OMP_NUM_THREADS=str(cores)),
                           check=True)
        d = json.loads(r.stdout.strip().splitlines()[-1])
        return {"value": d["mlups"], "unit": "MLUPS", "cores": d["threads"], "kind": "reference",
                "sample": f"{max_steps} full time steps of the {nx}x{ny}x{nz} box after {warmup} warm-up "
                          f"(reference CPU solver built from its sources, OpenMP)", "ms_step": d["ms_step"]}
    # C restatement (one thread)
    from oracle import oracle as O
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    from cases import BC
    op = O.make_params(nx, ny, nz, BC[bc], ALPHA=alpha)
    q = O.seeded_q(op, SEED, O.equilibrium_order(op), SIGMA)
    sim = O.OracleSim(op)
    sim.set(np.ones(V), np.zeros(3 * V), q)
    sim.step(warmup)
    t0 = time.perf_counter()
    sim.step(max_steps)
    dt = time.perf_counter() - t0
    return {"value": V * max_steps / dt / 1e6, "unit": "MLUPS", "cores": 1, "kind": "port",
            "sample": f"{max_steps} full time steps of the {nx}x{ny}x{nz} box (C restatement)",
            "ms_step": dt * 1e3 / max_steps}


REF_GPU_BUILD = {"periodic512": "b_p512", "slit64": "b_slit"}


def reference_gpu(workload, steps=10, warmup=3):
    """The reference's own FP64 CUDA solver (DeviceSolver<SimBC>, src/cuda,
    built from its sources by oracle/build_ref.py) on the same seeded
    workload, timed with CUDA events: the GPU baseline of the FP64 path."""
    from oracle import build_ref
    tag = REF_GPU_BUILD.get(workload)
    exe = build_ref.gpu_bench_path(tag) if tag else None
    if not exe or not os.path.exists(exe):
        return {"value": None, "error": "reference GPU build absent for this workload"}
    r = subprocess.run([exe, str(SEED), repr(S0), repr(SIGMA), str(warmup), str(steps)], capture_output=True,
                       text=True, timeout=900)
    d = json.loads(r.stdout.strip().splitlines()[-1])
    if "error" in d:
        return {"value": None, "error": d["error"][:300]}
    nx, ny, nz, *_ = WORKLOADS[workload]
    peak, _ = measured_peaks()
    return {"value": d["mlups"], "unit": "MLUPS", "dtype": "f64", "steps": steps, "ms_per_step": d["ms_step"],
            "ms_q_stage": d["ms_q"], "ms_lbm": d["ms_lbm"],
            "note": "reference src/cuda kernels (GpuQTensorStep + GpuComputeBodyForce + GpuCollideAndStream), "
                    "sm_100a build of its sources, default stream, CUDA events",
            "frac_at_368B": 368 * nx * ny * nz / (d["ms_step"] * 1e-3) / 1e9 / peak}


def ref_sample_steps(V, steps):
    """Steps of a bounded CPU sample: about half a minute of reference work."""
    return max(1, min(steps, 3 if V > 5e7 else 20 if V > 1e6 else 200))


def side_workloads(names, device, stream, steps=2000):
    """The other single-GPU solver workloads (channel and slit configurations),
    FP32, autotuned, device-timed: MLUPS and the whole step's HBM fraction."""
    peak, _ = measured_peaks()
    out = {}
    for w in names:
        nx, ny, nz, bc, alpha, _ = WORKLOADS[w]
        s, p = make_sim(w, "fp32", device)
        s.set_stream(stream.cuda_stream)
        s.init_seeded(SEED, S0, SIGMA)
        tuned = s.autotune(steps_per_trial=10)
        ms, _ = time_device(s, steps, 20, stream)
        s.close()
        out[f"{bc}_{nx}x{ny}x{nz}"] = {"value": p.V * steps / (ms * 1e3), "unit": "MLUPS", "steps": steps,
                                       "ms_per_step": ms / steps,
                                       "step_frac": BYTES_PER_CELL["fp32"] * p.V / (ms / steps * 1e-3) / 1e9 / peak,
                                       "shape": {k: tuned[k] for k in ("kernels", "tile_x", "tile_y", "zchunk")}}
    return out


def halo_bytes_per_step(nx, ny, precision):
    """Bytes one slab sends per step: the Q/u halo (2 faces x 8 components x
    2 planes) every step, the population halos (2 faces x 5 slots, in and
    out) every other step."""
    rb = 8 if precision == "fp64" else 4
    sb = {"fp64": 8, "fp32": 4, "fp16": 2}[precision]
    return nx * ny * (2 * 8 * 2 * rb + 2 * 5 * sb)


def make_slabs(workload, precision, device, kernels, tile, nslabs):
    import lbman3d_b200 as L
    nx, ny, nz, bc, alpha, _ = WORKLOADS[workload]
    p = L.Params(nx=nx, ny=ny, nz=nz, ALPHA=alpha)
    prec = {"fp64": L.Precision.FP64, "fp32": L.Precision.FP32, "fp16": L.Precision.FP16}[precision]
    return L.SlabBox(p, bc_for(bc), prec, nslabs=nslabs, kernels=kernels, devices=(device,), tile=tile), p


def slab_split(workload, precision, device, stream, kernels, tile, nslabs=2, steps=40, warmup=4):
    """The box as nslabs z-slabs on this one GPU, exchanging through
    lbman_slab_exchange on one stream: the cost of the decomposition's ghost
    planes, exchanges and extra launches, against the single box."""
    import torch
    sb, p = make_slabs(workload, precision, device, kernels, tile, nslabs)
    try:
        for s in sb.slabs:
            s.set_stream(stream.cuda_stream)
        sb.init_seeded(SEED, S0, SIGMA)
        sb.step(warmup)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        sb.step(steps)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1)
    finally:
        sb.close()
    return {"slabs": nslabs, "value": p.V * steps / (ms * 1e3), "unit": "MLUPS", "steps": steps,
            "ms_per_step": ms / steps, "halo_bytes_per_slab_step": halo_bytes_per_step(p.nx, p.ny, precision)}


def time_slab_ranks(a, workload, local, stream):
    """Strong scaling (--decomp slab): the box split into one z-slab per rank,
    exchanging over NCCL point-to-point operations (DistributedSlab)."""
    import torch
    import lbman3d_b200 as L
    nx, ny, nz, bc, alpha, _ = WORKLOADS[workload]
    p = L.Params(nx=nx, ny=ny, nz=nz, ALPHA=alpha)
    prec = {"fp64": L.Precision.FP64, "fp32": L.Precision.FP32, "fp16": L.Precision.FP16}[a.precision]
    kern = {"auto": L._native.KERNELS_AUTO, "split": L._native.KERNELS_SPLIT,
            "pair": L._native.KERNELS_SPLIT_PAIR}[a.kernels]
    tile = tuple(int(v) for v in a.tile.split(",")) if a.tile else None
    with torch.cuda.stream(stream):
        ds = L.DistributedSlab(p, bc_for(bc), prec, kern, tile=tile)
        try:
            ds.slab.init_seeded(SEED, S0, SIGMA)
            if a.kernels == "auto" and not tile:  # per slab; restores the state it advances
                ds.slab.autotune(steps_per_trial=8)
            ds.step(max(a.warmup, 3))
            l0 = ds.slab.launch_count()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            ds.step(a.steps)
            e1.record(stream)
            e1.synchronize()
            ms, launches = e0.elapsed_time(e1), ds.slab.launch_count() - l0
            d = ds.reduce(L._native.DIAG_FLOW)
        finally:
            ds.close()
    return ms, launches, d, halo_bytes_per_step(nx, ny, a.precision)


def time_ensemble_ranks(a, local, stream, world, rank, nboxes=96):
    """The batching workload spread over the ranks (--decomp ensemble): each
    rank advances its cell-balanced share of the 96 boxes (ShardedEnsemble),
    no exchange while stepping."""
    import torch
    import lbman3d_b200 as L
    boxes = L.draw_boxes(nboxes, seed=2024)
    ens = L.ShardedEnsemble(boxes, rank, world, L.Precision.FP32, device=local)
    try:
        ens.set_stream(stream.cuda_stream)
        ens.init_seeded(7)
        ens.autotune(steps_per_trial=3)
        ens.step(max(a.warmup, 3))
        ens.synchronize()
        l0 = ens.info()["launches"]
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ens.step(a.steps)
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1), ens.info()["launches"] - l0, sum(p.V for p, _ in boxes), len(ens)
    finally:
        ens.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="periodic512", choices=list(WORKLOADS))
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64", "fp16"])
    ap.add_argument("--error-steps", type=int, default=2000,
                    help="steps of the FP32/FP16 runs compared with the FP64 path")
    ap.add_argument("--no-extras", action="store_true", help="skip e2e, cpu baseline and variants")
    ap.add_argument("--kernels", default="auto", choices=["auto", "fused", "split", "pair"])
    ap.add_argument("--tile", default=None, help="tcx,tcy[,zchunk] of the z-marching kernels")
    ap.add_argument("--decomp", default="replicas", choices=["replicas", "slab", "ensemble"],
                    help="N > 1: one box per GPU (weak scaling), one box split into z-slabs (strong), or "
                         "the 96-box ensemble shared out over the GPUs (strong)")
    a = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    nx, ny, nz, bc, alpha, _ = WORKLOADS[a.workload]
    V = nx * ny * nz
    config = {"workload": f"{bc}_{nx}x{ny}x{nz}", "bc": bc, "zeta": alpha, "LAMBDA": 0.3, "advection": "centred",
              "init": f"seeded random director (seed {SEED}), S0={S0}, {SIGMA:g} Gaussian",
              "l2": "state larger than L2 (126 MB)" if V * BYTES_PER_CELL[a.precision] > 126e6
              else "state fits in L2", "parallelism": f"replicas x{a.gpus}"}

    if a.impl == "reference":
        if rank != 0:
            return
        n, w = ref_sample_steps(V, a.steps), min(a.warmup, 1)
        try:
            r = reference_cpu(a.workload, n, w)
        except (RuntimeError, subprocess.CalledProcessError, OSError) as e:
            print(json.dumps({"impl": "reference", "unavailable": str(e)[:300]}), flush=True)
            return
        line = {"impl": "reference", "metric": "MLUPS", "value": r["value"], "unit": "MLUPS", "n_gpus": a.gpus,
                "steps": n, "warmup": w, "ms_per_step": r["ms_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config,
                "cpu_baseline": {k: r[k] for k in ("value", "unit", "cores", "kind", "sample")},
                "e2e": {"value": r["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line), flush=True)
        return

    import torch
    import torch.distributed as dist
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        dist.init_process_group("nccl", init_method="env://", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    stream = torch.cuda.Stream(device=local)

    if a.decomp == "ensemble":
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        with ClockSampler(local) as clk:
            ms, launches, cells, mine = time_ensemble_ranks(a, local, stream, world, rank)
        ms = reduce_max(ms, world, "cuda")
        config = {"workload": "ensemble of 96 boxes (sides 24-96, periodic / slit, seed 2024)", "cells": cells,
                  "parallelism": f"boxes sharded x{world} (cell-balanced greedy)", "boxes_rank0": mine,
                  "l2": "state larger than L2 (126 MB)"}
        peak, peak_kind = measured_peaks()
        step_achieved = BYTES_PER_CELL["fp32"] * cells / (ms / a.steps * 1e-3) / 1e9
        line = {"metric": "MLUPS", "value": cells * a.steps / (ms * 1e3), "unit": "MLUPS", "n_gpus": world,
                "steps": a.steps, "warmup": max(a.warmup, 3), "ms_per_step": ms / a.steps, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": config,
                "gpu_launches": launches,
                "roofline": {"bound": "hbm", "achieved": step_achieved, "peak": peak * world, "unit": "GB/s",
                             "frac": step_achieved / (peak * world), "traffic": None, "peak_kind": peak_kind,
                             "kernel": "step (all boxes)", "step_bytes_per_cell": BYTES_PER_CELL["fp32"]},
                "clocks": clk.summary()}
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return

    if a.decomp == "slab":
        config["parallelism"] = f"z-slabs x{world}"
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        with ClockSampler(local) as clk:
            ms, launches, diag, hb = time_slab_ranks(a, a.workload, local, stream)
        ms = reduce_max(ms, world, "cuda")
        peak, peak_kind = measured_peaks()
        bpc = BYTES_PER_CELL[a.precision]
        step_achieved = bpc * V / (ms / a.steps * 1e-3) / 1e9
        line = {"metric": "MLUPS", "value": V * a.steps / (ms * 1e3), "unit": "MLUPS", "n_gpus": world,
                "steps": a.steps, "warmup": max(a.warmup, 3), "ms_per_step": ms / a.steps, "higher_is_better": True,
                "scaling": "strong", "vs_baseline": None,
                "dtype": {"fp32": "f32", "fp64": "f64", "fp16": "f32 (f16 storage)"}[a.precision],
                "data": "synthetic", "config": config, "gpu_launches": launches,
                "roofline": {"bound": "hbm", "achieved": step_achieved, "peak": peak * world, "unit": "GB/s",
                             "frac": step_achieved / (peak * world), "traffic": None, "peak_kind": peak_kind,
                             "kernel": "step (all slabs)", "step_bytes_per_cell": bpc},
                "halo_bytes_per_rank_step": hb, "mass": diag["mass"], "clocks": clk.summary()}
        if rank == 0:
            print(json.dumps(line), flush=True)
        if world > 1:
            dist.barrier()
            dist.destroy_process_group()
        return

    tile = tuple(int(v) for v in a.tile.split(",")) if a.tile else None
    sim, p = make_sim(a.workload, a.precision, local, a.kernels, tile)
    sim.set_stream(stream.cuda_stream)
    if a.kernels == "auto" and not tile:
        sim.init_seeded(SEED, S0, SIGMA)
        tuned = sim.autotune(steps_per_trial=8 if V > 5e7 else 10)
        config["autotuned"] = {k: tuned[k] for k in ("kernels", "tile_x", "tile_y", "zchunk", "trials")}
    sh = sim.shape()
    config["kernels"] = {1: "split", 2: "fused", 3: "split_pair"}[sh["kernels"]]
    config["tile"] = [sh["tile_x"], sh["tile_y"], sh["zchunk"]]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        ms, launches = time_device(sim, a.steps, max(a.warmup, 3), stream)
    ms = reduce_max(ms, world, "cuda")
    ms_step = ms / a.steps
    mlups = whole_job_rate(V, a.steps, world, ms)
    peak, peak_kind = measured_peaks()
    bpc = BYTES_PER_CELL[a.precision]
    step_achieved = bpc * V / (ms_step * 1e-3) / 1e9
    kern = kernel_breakdown(sim, config["kernels"], a.precision, V, stream, 30 if V > 5e7 else 200)
    dom = max(kern, key=lambda k: kern[k]["ms"])
    achieved = kern[dom]["bytes_per_cell"] * V / (kern[dom]["ms"] * 1e-3) / 1e9
    for k in kern:
        kern[k]["frac"] = kern[k]["bytes_per_cell"] * V / (kern[k]["ms"] * 1e-3) / 1e9 / peak
    line = {"metric": "MLUPS", "value": mlups, "unit": "MLUPS", "n_gpus": world, "steps": a.steps,
            "warmup": max(a.warmup, 3), "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": {"fp32": "f32", "fp64": "f64", "fp16": "f32 (f16 storage)"}[a.precision],
            "data": "synthetic", "config": config, "gpu_launches": launches,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": profile_traffic(config["workload"], a.precision, dom),
                         "peak_kind": peak_kind, "kernel": dom, "kernels": kern,
                         "step_bytes_per_cell": bpc, "step_achieved": step_achieved,
                         "step_frac": step_achieved / peak},
            "clocks": clk.summary()}
    if not a.no_extras:
        line["e2e"] = time_e2e(sim, p, 5, stream, world=world, device="cuda")
    sim.close()
    torch.cuda.empty_cache()
    if not a.no_extras and world == 1:  # single-GPU extras; at N > 1 every rank runs only the legs above
        line["error_vs_fp64"] = errors_vs_fp64(a.workload, ["fp32", "fp16"], local, a.error_steps)
        variants = {}
        for prec in ("fp64", "fp16", "fp32"):
            if prec == a.precision:
                continue
            s2, _ = make_sim(a.workload, prec, local)
            s2.set_stream(stream.cuda_stream)
            s2.init_seeded(SEED, S0, SIGMA)
            tuned2 = s2.autotune(steps_per_trial=3)
            n2 = max(100, a.steps // 2)
            ms2, _ = time_device(s2, n2, 10, stream)
            variants[prec] = {"value": V * n2 / (ms2 * 1e3), "unit": "MLUPS", "steps": n2,
                              "frac": BYTES_PER_CELL[prec] * V / (ms2 / n2 * 1e-3) / 1e9 / peak,
                              "shape": {k: tuned2[k] for k in ("kernels", "tile_x", "tile_y", "zchunk")}}
            s2.close()
            torch.cuda.empty_cache()
        line["variants"] = variants
        try:
            line["reference_gpu"] = reference_gpu(a.workload)
            if line["reference_gpu"].get("value") and "fp64" in variants:
                line["reference_gpu"]["fp64_speedup"] = variants["fp64"]["value"] / line["reference_gpu"]["value"]
        except Exception as e:  # reported, never required
            line["reference_gpu"] = {"value": None, "error": str(e)[:300]}
        line["other_workloads"] = side_workloads([w for w in ("slit64", "channel20") if w != a.workload], local,
                                                 stream)
        line["ensemble"] = ensemble_vs_sequential(local, stream)
        kern_id = {"split": 1, "split_pair": 3}.get(config["kernels"], 1)
        line["slab_split"] = slab_split(a.workload, a.precision, local, stream, kern_id, tuple(config["tile"]))
        line["slab_split"]["vs_single_box"] = line["slab_split"]["value"] / mlups
        torch.cuda.empty_cache()
        try:
            r = reference_cpu(a.workload, ref_sample_steps(V, a.steps), 1)
            line["cpu_baseline"] = {k: v for k, v in r.items() if k != "ms_step"}
        except Exception as e:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "unit": "MLUPS", "error": str(e)[:300]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
