"""Closure experiment: train the coarse-grid closure on box-filtered fine runs
and measure it against a held-out fine run and against the plain coarse solver.

    python -m lbman3d_b200.closure_experiment [--fine 256] [--factor 4] ...

Fine runs: FullyPeriodic, FP32, seeded random director (S0 = equilibrium
order, 1e-3 Gaussian), zeta = ALPHA.  The training runs advance together in
one ensemble (one box per training seed); every ``factor`` fine steps each
box's state is box-filtered onto the coarse grid straight from the device
(one coarse step = ``factor`` fine steps, coarse parameters from
closure.coarse_params).  Training is one-step pairs first, then rounds of
rollout ("pushforward") pairs: the corrected coarse run is advanced m steps
from a filtered snapshot with the current network, and the pair asks for the
correction that brings that drifted state back onto the filtered fine run
(``--push-m``, ``--push-iters``).  The held-out seed is the yardstick:

* short-time error: relative L2 error of coarse Q and u against the
  filtered fine run after n coarse steps from the same filtered start, for
  the corrected and the plain coarse solver;
* statistics over the rollout window: defect density, mean |u|, the
  kinetic-energy spectrum and the Q correlation length, relative to the
  filtered fine run, for both;
* cost: device time per simulated coarse step of the fine solver (factor
  steps) against the corrected coarse solver (network + step), CUDA events.

Training adds Gaussian noise (``--train-noise``, normalised units) to the
network inputs, which makes the corrected runs drift less.  Prints one JSON
object.  Fallback rule: the closure is reported ``usable``
only if every statistic is within ``--tolerance`` of the fine run; otherwise
the fine solver is the answer.
"""
from __future__ import annotations

import argparse
import json
import math
import time

import numpy as np


def _stats(sim, nbins):
    st = sim.statistics()
    E, _ = sim.velocity_spectrum(nbins)
    _, _, xi = sim.q_correlation(nbins)
    return {"defect_density": st["defect_density"], "mean_speed": st["mean_speed"], "xi": xi, "E": E}


def _mean_stats(rows):
    out = {k: float(np.mean([r[k] for r in rows])) for k in ("defect_density", "mean_speed", "xi")}
    out["E"] = np.mean([r["E"] for r in rows], axis=0)
    return out


def _rel(a, b):
    return abs(a - b) / max(abs(b), 1e-30)


def run(fine_n=256, factor=4, zeta=0.01, train_seeds=(11, 12, 13), test_seed=99, burn=2000, snaps=120,
        iters=3000, lr=1e-3, rollout=100, tolerance=0.05, train_noise=0.05, push_m=(), push_iters=2000,
        push_stride=2, log=print):
    import torch

    import lbman3d_b200 as L
    from lbman3d_b200 import closure as CL

    t0 = time.time()
    fp = L.Params(nx=fine_n, ny=fine_n, nz=fine_n, ALPHA=zeta)
    cp = CL.coarse_params(fp, factor)
    S0 = L.EquilibriumScalarOrder(fp)
    bc = L.FullyPeriodicConfig()
    nc = fine_n // factor
    nbins = nc // 2
    stream = torch.cuda.Stream()  # a capturable stream: the ensemble replays its steps from CUDA graphs
    res = {"fine_grid": [fine_n] * 3, "coarse_grid": [nc] * 3, "factor": factor, "zeta": zeta,
           "train_seeds": list(train_seeds), "test_seed": test_seed, "burn_in_steps": burn,
           "snapshots_per_seed": snaps, "train_iters": iters, "lr": lr, "train_input_noise": train_noise,
           "rollout_coarse_steps": rollout, "push_m": list(push_m), "push_iters": push_iters,
           "push_stride": push_stride,
           "coarse_params": {"TAUF": cp.TAUF, "GAMMA": cp.GAMMA, "L": cp.L, "ALPHA": cp.ALPHA}}

    fine = L.Simulation(fp, bc, L.Precision.FP32)
    coarse = L.Simulation(cp, bc, L.Precision.FP32)
    plain = L.Simulation(cp, bc, L.Precision.FP32)
    probe = L.Simulation(cp, bc, L.Precision.FP32)
    for s in (fine, coarse, plain, probe):
        s.set_stream(stream.cuda_stream)
    cl = CL.Closure(nc, nc, nc, seed=1)
    cl.set_options(train_noise=train_noise)

    # --- training data: the training runs advance together in one ensemble ------
    ens = L.Ensemble([(fp, bc)] * len(train_seeds), L.Precision.FP32, device=torch.cuda.current_device())
    ens.set_stream(stream.cuda_stream)
    ens.init_seeded_each(list(train_seeds), 1e-3)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ens.step(burn)
    for b in range(len(train_seeds)):
        cl.record_box(ens, b, b)
    for _ in range(snaps):
        ens.step(factor)
        for b in range(len(train_seeds)):
            cl.record_box(ens, b, b)
    e1.record(stream)
    e1.synchronize()
    res["ensemble"] = {"boxes": len(train_seeds), "cells": len(train_seeds) * fp.V,
                       "fine_steps": burn + snaps * factor, "ms": e0.elapsed_time(e1),
                       "mlups": len(train_seeds) * fp.V * (burn + snaps * factor) / (e0.elapsed_time(e1) * 1e3)}
    ens.close()
    cl.build_targets(coarse)
    res["dataset"] = dict(zip(("snapshots", "pairs"), cl.dataset()))
    log(f"data ready: {res['dataset']} ({time.time() - t0:.1f} s)")

    # --- training: one-step pairs, then rounds of rollout pairs ------------------
    e0.record(stream)
    first, last = cl.train(iters, lr=lr, seed=7)
    e1.record(stream)
    e1.synchronize()
    res["train"] = {"loss_first_tenth": first, "loss_last_tenth": last,
                    "ms_per_iteration": e0.elapsed_time(e1) / iters, "rounds": []}
    log(f"trained: loss {first:.4g} -> {last:.4g} ({time.time() - t0:.1f} s)")
    for r, m in enumerate(push_m):
        added = cl.add_rollout_pairs(coarse, int(m), push_stride)
        first, last = cl.train(push_iters, lr=lr * 0.5, seed=100 + r)
        res["train"]["rounds"].append({"m": int(m), "pairs_added": added, "pairs": cl.dataset()[1],
                                       "loss_first_tenth": first, "loss_last_tenth": last})
        log(f"rollout round m={m}: +{added} pairs, loss {first:.4g} -> {last:.4g} ({time.time() - t0:.1f} s)")

    # --- held-out run: filtered fine trajectory --------------------------------
    n0, _ = cl.dataset()
    fine.init_seeded(test_seed, S0, 1e-3)
    fine.step(burn)
    cl.record(fine, new_trajectory=True)
    fine_stats, fine_fields = [], []
    fine_ms = 0.0
    for t in range(rollout):
        e0.record(stream)
        fine.step(factor)
        e1.record(stream)
        e1.synchronize()
        fine_ms += e0.elapsed_time(e1)
        cl.record(fine)
    fine_ms /= rollout
    for t in range(rollout + 1):
        cl.load_snapshot(n0 + t, probe)
        if t >= rollout // 2:
            fine_stats.append(_stats(probe, nbins))
        if t in (1, 5, 20, rollout):
            fine_fields.append((t, probe.download()))

    # --- corrected and plain coarse runs from the same filtered start -------------
    cl.load_snapshot(n0, coarse)
    cl.load_snapshot(n0, plain)
    cl_stats, pl_stats, errs = [], [], []
    targets = dict(fine_fields)
    ms_cl = ms_pl = 0.0
    for t in range(1, rollout + 1):
        e0.record(stream)
        cl.step(coarse, 1)
        e1.record(stream)
        e1.synchronize()
        ms_cl += e0.elapsed_time(e1)
        e0.record(stream)
        plain.step(1)
        e1.record(stream)
        e1.synchronize()
        ms_pl += e0.elapsed_time(e1)
        if t >= rollout // 2 + 1:
            cl_stats.append(_stats(coarse, nbins))
            pl_stats.append(_stats(plain, nbins))
        if t in targets:
            ref = targets[t]
            row = {"step": t}
            for name, sim in (("closure", coarse), ("plain", plain)):
                o = sim.download()
                for f in ("q", "u"):
                    row[f"{name}_{f}"] = float(np.linalg.norm(o[f] - ref[f]) / np.linalg.norm(ref[f]))
            errs.append(row)
    res["short_time_relative_l2"] = errs

    F, Cc, P = _mean_stats(fine_stats), _mean_stats(cl_stats), _mean_stats(pl_stats)
    kmax = max(2, nc // 4)

    def spec_err(E):
        return float(np.linalg.norm(E[1:kmax] - F["E"][1:kmax]) / np.linalg.norm(F["E"][1:kmax]))

    res["statistics"] = {
        "window_coarse_steps": [rollout // 2, rollout],
        "fine_filtered": {k: F[k] for k in ("defect_density", "mean_speed", "xi")},
        "closure": {k: Cc[k] for k in ("defect_density", "mean_speed", "xi")},
        "plain_coarse": {k: P[k] for k in ("defect_density", "mean_speed", "xi")},
        "rel_err_closure": {"defect_density": _rel(Cc["defect_density"], F["defect_density"]),
                            "mean_speed": _rel(Cc["mean_speed"], F["mean_speed"]),
                            "xi": _rel(Cc["xi"], F["xi"]), "spectrum_l2": spec_err(Cc["E"])},
        "rel_err_plain": {"defect_density": _rel(P["defect_density"], F["defect_density"]),
                          "mean_speed": _rel(P["mean_speed"], F["mean_speed"]),
                          "xi": _rel(P["xi"], F["xi"]), "spectrum_l2": spec_err(P["E"])},
        "spectrum_shells_compared": [1, kmax - 1],
    }
    res["cost"] = {"fine_ms_per_coarse_step": fine_ms, "closure_ms_per_coarse_step": ms_cl / rollout,
                   "plain_coarse_ms_per_step": ms_pl / rollout,
                   "speedup_vs_fine": fine_ms / (ms_cl / rollout)}
    worst = max(res["statistics"]["rel_err_closure"].values())
    res["usable"] = bool(worst <= tolerance)
    res["fallback"] = "none" if res["usable"] else "fine solver (closure statistics outside tolerance)"
    res["tolerance"] = tolerance
    res["wall_s"] = time.time() - t0
    for s in (fine, coarse, plain, probe):
        s.close()
    cl.close()
    return res


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--fine", type=int, default=256)
    ap.add_argument("--factor", type=int, default=4)
    ap.add_argument("--zeta", type=float, default=0.01)
    ap.add_argument("--burn", type=int, default=2000)
    ap.add_argument("--snaps", type=int, default=120)
    ap.add_argument("--iters", type=int, default=3000)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--rollout", type=int, default=100)
    ap.add_argument("--seeds", type=int, default=3)
    ap.add_argument("--tolerance", type=float, default=0.05)
    ap.add_argument("--train-noise", type=float, default=0.05,
                    help="std of Gaussian noise on the normalised inputs while training")
    ap.add_argument("--push-m", default="", help="comma-separated rollout lengths of the pushforward rounds")
    ap.add_argument("--push-iters", type=int, default=2000)
    ap.add_argument("--push-stride", type=int, default=2)
    a = ap.parse_args(argv)
    import sys
    push = tuple(int(v) for v in a.push_m.split(",") if v.strip())
    res = run(a.fine, a.factor, a.zeta, tuple(range(11, 11 + a.seeds)), 99, a.burn, a.snaps, a.iters, a.lr,
              a.rollout, a.tolerance, a.train_noise, push, a.push_iters, a.push_stride,
              log=lambda m: print(m, file=sys.stderr, flush=True))
    print(json.dumps(res))


if __name__ == "__main__":
    main()
