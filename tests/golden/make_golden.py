"""Generate the golden parity fixtures in tests/golden/*.npz.

Each fixture holds the input fields of one small case and the fields the
reference's own CPU solver produced from them after the listed numbers of
steps.  The reference runs as oracle/_ref/<build>/ref_driver, compiled from
the reference sources by oracle/build_ref.py (this container only: the
reference tree is not present on GPU machines, so the fixtures are
committed).

    python tests/golden/make_golden.py            # all cases
    python tests/golden/make_golden.py periodic_p8
"""
from __future__ import annotations

import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

from cases import BC, CASES, GRID, PHYS, UPWIND  # noqa: E402
from oracle import build_ref  # noqa: E402
from oracle import oracle as O  # noqa: E402

SNAP_FIELDS = [("rho", 1), ("u", 3), ("q", 5), ("f", 15), ("force", 3), ("sigma", 5), ("tau", 3),
               ("order", 1), ("director", 3)]


def case_params(build: str, bc: str) -> O.Params:
    nx, ny, nz = GRID[build]
    return O.make_params(nx, ny, nz, BC[bc], O.UPWIND if build in UPWIND else O.CENTRED,
                         **PHYS[build])


def case_inputs(p: O.Params, init: str, seed: int):
    V = p.nx * p.ny * p.nz
    S0 = O.equilibrium_order(p)
    q = O.seeded_q(p, seed, S0, 1e-3)
    rng = np.random.default_rng(seed)
    rho = np.ones(V)
    u = np.zeros(3 * V)
    force = None
    if init == "perturbed":
        rho = 1.0 + 0.01 * rng.standard_normal(V)
        u = 0.01 * rng.standard_normal(3 * V)
    elif init.startswith("force:"):
        force = np.zeros(3 * V)
        force[:V] = float(init.split(":")[1])
    elif init != "baseline":
        raise ValueError(init)
    return rho, u, q, force


def read_snapshots(path: str, V: int, nsnap: int):
    raw = open(path, "rb").read()
    off = 0
    snaps = []
    for _ in range(nsnap):
        step = int(np.frombuffer(raw, np.int64, 1, off)[0]); off += 8
        s = {"step": step}
        for name, k in SNAP_FIELDS:
            s[name] = np.frombuffer(raw, np.float64, k * V, off).copy(); off += 8 * k * V
        diag = np.frombuffer(raw, np.float64, 9, off).copy(); off += 72
        s["free_energy"] = diag[0]
        s["log"] = diag[1:]
        s["defect_faces"], s["disclinations"] = np.frombuffer(raw, np.int64, 2, off).tolist(); off += 16
        snaps.append(s)
    assert off == len(raw), (off, len(raw))
    return snaps


def make(name: str) -> str:
    build, bc, mode, init, snaps = CASES[name]
    exe = build_ref.driver_path(build)
    if not os.path.exists(exe):
        build_ref.build(build, build_ref.REF_BUILDS[build])
    p = case_params(build, bc)
    V = p.nx * p.ny * p.nz
    rho, u, q, force = case_inputs(p, init, seed=sum(map(ord, name)))
    with tempfile.TemporaryDirectory() as td:
        fin, fout = os.path.join(td, "in.bin"), os.path.join(td, "out.bin")
        with open(fin, "wb") as fh:
            fh.write(np.int64(V).tobytes())
            fh.write(np.int32(0).tobytes())
            fh.write(np.int32(force is not None).tobytes())
            for a in (rho, u, q) + ((force,) if force is not None else ()):
                fh.write(np.ascontiguousarray(a, np.float64).tobytes())
        subprocess.run([exe, bc, mode, fin, fout] + [str(s) for s in snaps], check=True,
                       env=dict(os.environ, LBMAN_REF_THREADS="1"))
        out = read_snapshots(fout, V, len(snaps))
    arrays = dict(grid=np.array([p.nx, p.ny, p.nz]), faces=np.array(repr(BC[bc])),
                  phys=np.array(repr(PHYS[build])), upwind=np.array(build in UPWIND),
                  mode=np.array(mode), bc=np.array(bc), steps=np.array(snaps),
                  in_rho=rho, in_u=u, in_q=q,
                  in_force=force if force is not None else np.zeros(0))
    for k, s in enumerate(out):
        for key, val in s.items():
            arrays[f"s{k}_{key}"] = np.asarray(val)
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **arrays)
    return path


def main(argv):
    names = argv or list(CASES)
    for n in names:
        print("wrote", make(n))


if __name__ == "__main__":
    main(sys.argv[1:])
