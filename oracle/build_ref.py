"""Build recipe for oracle/_ref: the reference's own CPU solver, compiled from
its sources where they lie (never copied; the reference's src/ directory is
taken from $LBMAN_REFERENCE_SRC, by default /root/reference/src), with a
generated params.h/sim_config.h first on the include path -- the shadowing
the reference's own tests use (tests/CMakeLists.txt:3-8).

TEST INFRASTRUCTURE ONLY.  Each build is one compile-time parameter set
(the reference fixes grid size and physics constants at compile time); the
boundary configuration is chosen at run time by ref_driver.cc.

    python oracle/build_ref.py            # builds every set in REF_BUILDS
    python oracle/build_ref.py --list

Outputs: oracle/_ref/<tag>/ref_driver (plus the generated headers), and
oracle/_ref/<tag>/dropin_check for the DROPIN_BUILDS sets (the reference's
solver classes beside include/lbman3d_dropin.hpp, linked against the built
lbman3d_b200/liblbman3d_b200.so).
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SRC = os.environ.get("LBMAN_REFERENCE_SRC", "/root/reference/src")
OUT = os.path.join(HERE, "_ref")

# Physics defaults of src/params.h:36-112.
DEFAULTS = dict(DT=1.0, kDensity=1.0, TAUF=2.5, L=0.06, A=0.0, B=-0.3, C=0.3,
                LAMBDA=0.3, GAMMA=0.34, ALPHA=0.023, MU=0.0, NOISE=0.05)

# Compile-time parameter sets.  Grids are small (parity fixtures) except the
# CPU-baseline builds, which match the benchmark workloads.
REF_BUILDS = {
    # golden fixtures
    "g_p8": dict(nx=8, ny=8, nz=8),
    "g_678": dict(nx=6, ny=7, nz=8, ALPHA=0.02, MU=0.01),
    "g_678_up": dict(nx=6, ny=7, nz=8, ALPHA=0.02, advection="Upwind"),
    "g_thin": dict(nx=1, ny=5, nz=6),
    "g_unit": dict(nx=5, ny=5, nz=5, DT=0.05, TAUF=1.5 * 0.05, L=0.01, ALPHA=0.04),
    "g_lbm": dict(nx=5, ny=16, nz=5, TAUF=0.9330127018922193, ALPHA=0.0),
    # CPU baselines at the benchmark workloads (threads from the environment)
    "b_slit": dict(nx=64, ny=256, nz=256, ALPHA=0.01),
    "b_channel": dict(nx=20, ny=100, nz=100, ALPHA=0.01),
    "b_p32": dict(nx=32, ny=32, nz=32),
    "b_p512": dict(nx=512, ny=512, nz=512, ALPHA=0.01),
}

# Parameter sets of the C++ drop-in check (dropin_check.cc, linked against
# the built liblbman3d_b200.so).
DROPIN_BUILDS = {
    "d_box": dict(nx=10, ny=12, nz=8, ALPHA=0.02, MU=0.01),
}


def hexf(v: float) -> str:
    return float(v).hex()


def params_h(cfg: dict) -> str:
    p = dict(DEFAULTS)
    p.update({k: v for k, v in cfg.items() if k in DEFAULTS})
    lines = [
        "// Generated by oracle/build_ref.py -- shadows src/params.h.",
        "#ifndef LBM_AN_PARAMS_H_", "#define LBM_AN_PARAMS_H_",
        "#include <cstdlib>", "#include <omp.h>",
        "inline int lbman_ref_threads() {",
        "  const char* s = std::getenv(\"LBMAN_REF_THREADS\");",
        "  return (s && std::atoi(s) > 0) ? std::atoi(s) : omp_get_max_threads();",
        "}",
        "namespace Params {",
        "    static constexpr double kCs2Inv = 3.0;",
        "    static constexpr double kCs2InvTimes2 = 6.0;",
        "    static constexpr double kCs4Inv = 9.0;",
        "    static constexpr double khalfCs2Inv = 1.5;",
        "    static constexpr double khalfCs4Inv = 4.5;",
        f"    inline constexpr int nx = {int(cfg['nx'])};",
        f"    inline constexpr int ny = {int(cfg['ny'])};",
        f"    inline constexpr int nz = {int(cfg['nz'])};",
        "    inline const int kNumOMPThreads = lbman_ref_threads();",
        "    inline constexpr double DX = 1.0, DY = 1.0, DZ = 1.0;",
        f"    inline constexpr double DT = {hexf(p['DT'])};",
        f"    inline constexpr double kDensity = {hexf(p['kDensity'])};",
        f"    inline constexpr double TAUF = {hexf(p['TAUF'])};",
        "    inline constexpr double omega         = 1.0 - DT / TAUF;",
        "    inline constexpr double omega_prime   = DT / TAUF;",
        "    inline constexpr double omega_forcing = 1.0 - DT / 2.0 / TAUF;",
        f"    inline constexpr double L = {hexf(p['L'])};",
        f"    inline constexpr double A = {hexf(p['A'])};",
        f"    inline constexpr double B = {hexf(p['B'])};",
        f"    inline constexpr double C = {hexf(p['C'])};",
        f"    inline constexpr double LAMBDA = {hexf(p['LAMBDA'])};",
        f"    inline constexpr double GAMMA = {hexf(p['GAMMA'])};",
        f"    inline constexpr double ALPHA = {hexf(p['ALPHA'])};",
        f"    inline constexpr double MU = {hexf(p['MU'])};",
        f"    inline constexpr double NOISE = {hexf(p['NOISE'])};",
        "    inline constexpr double kLidVelocity = 0.0;",
        "    inline constexpr double kinematicViscosity = kDensity / kCs2Inv * (TAUF - 0.5 * DT);",
        "    inline constexpr bool kDebugLogging = false;",
        "    inline constexpr bool kTrackNematicEnergy = false;",
        "}", "#endif",
    ]
    return "\n".join(lines) + "\n"


def sim_config_h(cfg: dict) -> str:
    adv = cfg.get("advection", "Centred")
    bc = cfg.get("bc", "FullyPeriodicConfig")
    extra = []
    if bc == "SlitFreeSlipConfig":  # the reference's SlitConfig (src/sim_config.h:19-27)
        extra = ["struct SlitFreeSlipConfig {",
                 "    using XLo = WallSpec<Neumann, SpecularReflection>;",
                 "    using XHi = WallSpec<Neumann, SpecularReflection>;",
                 "    using YLo = WallSpec<Periodic, Periodic>;", "    using YHi = WallSpec<Periodic, Periodic>;",
                 "    using ZLo = WallSpec<Periodic, Periodic>;", "    using ZHi = WallSpec<Periodic, Periodic>;",
                 "};"]
    return "\n".join([
        "// Generated by oracle/build_ref.py -- shadows src/sim_config.h.",
        "#ifndef LBM_AN_SIM_CONFIG_H_", "#define LBM_AN_SIM_CONFIG_H_",
        "#include \"boundary.h\"", "#include \"qtensor_types.h\""] + extra + [
        f"using SimBC = {bc};",
        f"inline constexpr Advection kQAdvection = Advection::{adv};",
        "inline constexpr int kNumSteps = 1;", "inline constexpr int kSaveInterval = 1;",
        "#endif", ""])


def build(tag: str, cfg: dict, verbose: bool = False) -> str:
    if not os.path.isdir(REF_SRC):
        raise FileNotFoundError(f"{REF_SRC} is not present; oracle/_ref cannot be rebuilt here")
    d = os.path.join(OUT, tag)
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "params.h"), "w") as fh:
        fh.write(params_h(cfg))
    with open(os.path.join(d, "sim_config.h"), "w") as fh:
        fh.write(sim_config_h(cfg))
    # analysis/defect_finder.h includes vtkhdf_writer.h (HDF5) but uses none of it.
    with open(os.path.join(d, "vtkhdf_writer.h"), "w") as fh:
        fh.write("// empty stand-in: nothing from the HDF5 writer is used by the driver\n#pragma once\n")
    with open(os.path.join(d, "config.json"), "w") as fh:
        json.dump(dict(DEFAULTS, **cfg), fh, indent=1, sort_keys=True)
    exe = os.path.join(d, "ref_driver")
    # The project's seeded initial condition (orc_seeded_q), for the bench mode.
    gen = os.path.join(d, "lbman_oracle.o")
    subprocess.run(["gcc", "-std=c11", "-O2", "-ffp-contract=off", "-fopenmp", "-c", os.path.join(HERE, "lbman_oracle.c"),
                    "-o", gen], check=True)
    srcs = [os.path.join(HERE, "ref_driver.cc")] + [
        os.path.join(REF_SRC, s) for s in
        ("fluid_fields.cc", "qtensor_fields.cc", "analysis_fields.cc", "analysis/defect_fields.cc")]
    # The reference's release flags (CMakeLists.txt:59-60).
    cmd = ["g++", "-std=c++23", "-O3", "-DNDEBUG", "-fopenmp", "-w",
           "-I", d, "-I", REF_SRC, "-I", HERE, "-o", exe] + srcs + [gen, "-lm"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return exe


# Parameter sets of the reference's own CUDA solver timing (ref_gpu_bench.cu):
# the reference's src/cuda sources compiled for sm_100a.
GPU_BUILDS = {
    "b_p512": dict(nx=512, ny=512, nz=512, ALPHA=0.01),
    "b_slit": dict(nx=64, ny=256, nz=256, ALPHA=0.01, bc="SlitFreeSlipConfig"),
}


def gpu_bench_path(tag: str) -> str:
    return os.path.join(OUT, tag + "_gpu", "ref_gpu_bench")


def build_gpu(tag: str, cfg: dict, verbose: bool = False) -> str:
    """ref_gpu_bench for one parameter set: the reference's DeviceFields /
    DeviceSolver / kernels (src/cuda), nvcc for sm_100a with -DNDEBUG (the
    reference's release flags; its device-side index asserts compiled out)."""
    if not os.path.isdir(REF_SRC):
        raise FileNotFoundError(f"{REF_SRC} is not present; oracle/_ref cannot be rebuilt here")
    d = os.path.join(OUT, tag + "_gpu")
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "params.h"), "w") as fh:
        fh.write(params_h(cfg))
    with open(os.path.join(d, "sim_config.h"), "w") as fh:
        fh.write(sim_config_h(cfg))
    gen = os.path.join(d, "lbman_oracle.o")
    subprocess.run(["gcc", "-std=c11", "-O2", "-ffp-contract=off", "-fopenmp", "-c", os.path.join(HERE, "lbman_oracle.c"),
                    "-o", gen], check=True)
    exe = gpu_bench_path(tag)
    srcs = [os.path.join(HERE, "ref_gpu_bench.cu"), os.path.join(REF_SRC, "cuda", "device_fields.cu"),
            os.path.join(REF_SRC, "cuda", "device_solver.cu"), os.path.join(REF_SRC, "fluid_fields.cc"),
            os.path.join(REF_SRC, "qtensor_fields.cc")]
    cmd = [os.environ.get("NVCC", "nvcc"), "-gencode", "arch=compute_100a,code=sm_100a", "-std=c++20", "-O3",
           "-DNDEBUG", "-DSIM_WITH_CUDA", "-w", "-Xcompiler", "-fopenmp", "-I", d, "-I", REF_SRC,
           "-I", os.path.join(REF_SRC, "cuda"), "-I", HERE, "-o", exe] + srcs + [gen, "-lgomp"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return exe


def build_dropin(tag: str, cfg: dict, verbose: bool = False) -> str:
    """dropin_check for one parameter set; needs lbman3d_b200/liblbman3d_b200.so."""
    d = os.path.join(OUT, tag)
    os.makedirs(d, exist_ok=True)
    with open(os.path.join(d, "params.h"), "w") as fh:
        fh.write(params_h(cfg))
    with open(os.path.join(d, "sim_config.h"), "w") as fh:
        fh.write(sim_config_h(cfg))
    root = os.path.dirname(HERE)
    pkg = os.path.join(root, "lbman3d_b200")
    if not os.path.exists(os.path.join(pkg, "liblbman3d_b200.so")):
        raise FileNotFoundError("build lbman3d_b200 first (python -m lbman3d_b200.build)")
    exe = os.path.join(d, "dropin_check")
    srcs = [os.path.join(HERE, "dropin_check.cc")] + [
        os.path.join(REF_SRC, s) for s in ("fluid_fields.cc", "qtensor_fields.cc")]
    cmd = ["g++", "-std=c++23", "-O3", "-DNDEBUG", "-fopenmp", "-w",
           "-I", d, "-I", REF_SRC, "-I", os.path.join(root, "include"), "-o", exe] + srcs + [
           "-L", pkg, "-llbman3d_b200", "-Wl,-rpath,$ORIGIN/../../../lbman3d_b200"]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return exe


def dropin_path(tag: str) -> str:
    return os.path.join(OUT, tag, "dropin_check")


def driver_path(tag: str) -> str:
    return os.path.join(OUT, tag, "ref_driver")


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("tags", nargs="*")
    ap.add_argument("--list", action="store_true")
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args(argv)
    if a.list:
        for k, v in REF_BUILDS.items():
            print(k, v)
        return 0
    tags = a.tags or list(REF_BUILDS) + list(DROPIN_BUILDS) + [t + "_gpu" for t in GPU_BUILDS]
    for t in tags:
        if t.endswith("_gpu") and t[:-4] in GPU_BUILDS:
            build_gpu(t[:-4], GPU_BUILDS[t[:-4]], a.v)
            print("built", gpu_bench_path(t[:-4]))
        elif t in DROPIN_BUILDS:
            build_dropin(t, DROPIN_BUILDS[t], a.v)
            print("built", dropin_path(t))
        else:
            build(t, REF_BUILDS[t], a.v)
            print("built", driver_path(t))
    return 0


if __name__ == "__main__":
    sys.exit(main())
