"""Build lbman3d_b200/liblbman3d_b200.so (sm_100a) with nvcc, in tree.

    python -m lbman3d_b200.build [--force] [-v]

Translation units and their flags:
  kernels_f64.cu  --fmad=false  (FP64 path, bitwise parity with the reference)
  kernels_f32.cu  default contraction (FP32 path)
  kernels_f16.cu  default contraction (FP16 population storage)
  api.cu          host C ABI
  ens_api.cu      ensemble runner
  noalloc.cu      allocation-free flow diagnostics
  stats.cu        spectrum / correlation / speed statistics (links cuFFT)
Objects go to lbman3d_b200/_build/ (git-ignored).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIB = os.path.join(PKG, "liblbman3d_b200.so")
ROOT = os.path.dirname(PKG)
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
                 "-I", CSRC, "-I", INCLUDE]

UNITS = {
    "kernels_f64.cu": ["--fmad=false"],
    "kernels_f32.cu": [],
    "kernels_f16.cu": [],
    "kernels_ens.cu": [],
    "kernels_ens_f64.cu": ["--fmad=false"],
    "api.cu": [],
    "ens_api.cu": [],
    "noalloc.cu": [],
    "stats.cu": [],
    "closure_api.cu": [],
    "defects.cu": [],
}


def _sources_for(unit: str):
    deps = [os.path.join(CSRC, unit)]
    deps += [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    deps += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return deps


def _stale(target: str, deps) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    units = [u for u in UNITS if os.path.exists(os.path.join(CSRC, u))]
    jobs = []
    objs = []
    for u in units:
        obj = os.path.join(BUILD, u.replace(".cu", ".o"))
        objs.append(obj)
        if force or _stale(obj, _sources_for(u)):
            cmd = [NVCC] + COMMON + UNITS[u] + ["-c", os.path.join(CSRC, u), "-o", obj]
            jobs.append(cmd)
    if jobs:
        with cf.ThreadPoolExecutor(max_workers=len(jobs)) as ex:
            futs = [ex.submit(subprocess.run, cmd, capture_output=True, text=True) for cmd in jobs]
            for cmd, fut in zip(jobs, futs):
                r = fut.result()
                if verbose:
                    print(" ".join(cmd))
                if r.returncode != 0:
                    sys.stderr.write(r.stdout + r.stderr)
                    raise RuntimeError("nvcc failed: " + " ".join(cmd))
    if force or jobs or not os.path.exists(LIB):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart", "-lcufft"]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(a.force, a.v))
