#!/usr/bin/env python3
"""Builds the reference-kernel harness (test and baseline infrastructure).

Reads the reference's own kernel sources from --reference (the
petbab/fluid-simulation checkout), writes shimmed build-time copies into
oracle/_ref/<variant>/src (git-ignored, never committed) and compiles them
with oracle/refpath/*.cu into oracle/_ref/<variant>/librefpath.so.

Shims (the sources do not build outside KTT/NVRTC as they are):
  * `#include KERNEL_PATH(/common.cuh)` / `CUDA_PATH(...)` token pasting is
    rejected by the GCC preprocessor -> plain relative includes;
  * compile-time physics constants (PARTICLE_RADIUS, STIFFNESS, VISCOSITY,
    SURFACE_TENSION_ALPHA, GRAVITY) -> the variant's values;
  * `#pragma unroll <name>_u_n` needs a constant expression -> constexpr
    variables defined by oracle/refpath/ref_kernels.cu before the include.
Every replaced line is asserted to exist so a changed reference fails loudly.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
OUT = HERE / "_ref"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++20", *ARCH, "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr", "-w"]

KERNEL_FILES = ["rebuild_n_search.cu", "compute_neighbor_list.cu", "compute_rho_p.cu",
                "compute_pressure_accel_n_normal.cu", "compute_non_pressure_accel.cu", "update_positions.cu",
                "compute_boundary_mass.cu"]
FAMILIES = {1: "rebuild_fluid", 2: "rebuild_boundary", 3: "nlist", 4: "rho", 5: "pressure", 6: "nonpressure",
            7: "update", 8: "bmass"}

REF_DEFAULT = dict(r=0.02, k=0.1, nu=0.001, alpha=0.13, g=(0.0, -9.81, 0.0),
                   force="([](float4) {return make_float4(0.f); })", cell_mult="1.0",
                   min_dt=1e-5, max_dt=5e-4, cfl=0.4, np_max=0.015)

# Variants: one build per (particle counts, constants, frozen KTT parameters).
VARIANTS = {
    # 1,048,576-particle tilting box; frozen config of the largest shipped
    # scene (measurements/configs/BIG_falling.json: all blocks 32,
    # TABLE_SIZE_MULT 4, CELL_SIZE_MULT 1.0, neighbour lists, no smem)
    "large_tilting": dict(n=1048576, nb=0, r=0.004, k=("textbook", 1000.0), nu=0.01, max_dt=5e-4, cfl=0.0, table_mult=4, block=32),
    # the same scene at the other block sizes of the reference tuner's space
    # (step_tuner.cuh:331: 32, 64, 128, 256, 512)
    # (the reference arm of bench.py reports the fastest)
    **{f"large_tilting_b{b}": dict(n=1048576, nb=0, r=0.004, k=("textbook", 1000.0), nu=0.01, max_dt=5e-4, cfl=0.0,
                                   table_mult=4, block=b) for b in (64, 128, 256, 512)},
    # 32^3 dam break with walls (dragon_settled.json: blocks 32, TABLE_SIZE_MULT 32)
    "dam_break": dict(n=32768, nb=7802, r=0.01, k=("textbook", 1000.0), nu=0.01, max_dt=1e-3, cfl=0.0, table_mult=32, block=32),
    # mesh obstacle: 64 x 96 x 64 fluid block (r = 0.005) over a level-4
    # icosphere in a 1 m cube; 64,276 wall + sphere particles; CFL 0.4, dt cap 1e-3
    "mesh_obstacle": dict(n=393216, nb=64276, r=0.005, k=("textbook", 1000.0), nu=0.01, max_dt=1e-3, cfl=0.4,
                          table_mult=4, block=32),
    # golden fixtures (2048 particles)
    "fixture_surface": dict(n=2048, nb=0, force="([](float4 pos) { return make_float4(0., 9.81f, 0., 0.); })",
                            table_mult=8, block=64),
    "fixture_tilting": dict(n=2048, nb=0, table_mult=16, block=32),
    "fixture_dambreak": dict(n=2048, nb=3202, r=0.01, k=("textbook", 1000.0), nu=0.01, max_dt=1e-3, cfl=0.0, table_mult=4,
                             block=32),
}


def textbook_stiffness(k: float, r: float) -> float:
    """k * h^6 with h = 4r (float32 of the double product, as the presets compute it)."""
    import numpy as np

    rd = float(np.float32(r))
    return float(np.float32(k * (4.0 * rd) ** 6))


def bit_ceil(x: int) -> int:
    return 1 if x <= 1 else 1 << (x - 1).bit_length()


def replace_once(text: str, old: str, new: str, what: str) -> str:
    if old not in text:
        raise SystemExit(f"build_ref: expected text not found in {what}: {old!r}")
    return text.replace(old, new, 1)


def shim_sources(ref: Path, dst: Path):
    dst.mkdir(parents=True, exist_ok=True)
    kdir = ref / "src" / "cuda" / "tuning" / "kernels"
    cdir = ref / "src" / "cuda"
    for f in KERNEL_FILES:
        t = (kdir / f).read_text()
        t = replace_once(t, "#define KERNEL_PATH(file) <KERNEL_DIR ## file>", "", f)
        t = replace_once(t, "#include KERNEL_PATH(/common.cuh)", '#include "common.cuh"', f)
        if f == "compute_rho_p.cu":
            t = replace_once(t, "static constexpr float STIFFNESS = 0.1f;",
                             "static constexpr float STIFFNESS = REF_STIFFNESS;", f)
        if f == "compute_non_pressure_accel.cu":
            t = replace_once(t, "static constexpr float4 GRAVITY{0, -9.81f, 0, 0};",
                             "static constexpr float4 GRAVITY{REF_GX, REF_GY, REF_GZ, 0};", f)
            t = replace_once(t, "static constexpr float VISCOSITY = 0.001f;",
                             "static constexpr float VISCOSITY = REF_VISCOSITY;", f)
            t = replace_once(t, "static constexpr float SURFACE_TENSION_ALPHA = 0.13f;",
                             "static constexpr float SURFACE_TENSION_ALPHA = REF_SURFACE_TENSION;", f)
        (dst / f).write_text(t)
    t = (kdir / "common.cuh").read_text()
    t = replace_once(t, "#define CUDA_DIR KERNEL_DIR/../..", "", "common.cuh")
    t = replace_once(t, "#define CUDA_PATH(file) <CUDA_DIR ## file>", "", "common.cuh")
    t = replace_once(t, "#include CUDA_PATH(/math.cuh)", '#include "math.cuh"', "common.cuh")
    t = replace_once(t, "#include CUDA_PATH(/util.cuh)", '#include "util.cuh"', "common.cuh")
    t = replace_once(t, "#include CUDA_PATH(/SPH/kernel.cuh)", '#include "kernel.cuh"', "common.cuh")
    t = replace_once(t, "#include CUDA_PATH(/nsearch/morton.cuh)", '#include "morton.cuh"', "common.cuh")
    t = replace_once(t, "static constexpr float PARTICLE_RADIUS = 0.02f;",
                     "static constexpr float PARTICLE_RADIUS = REF_PARTICLE_RADIUS;", "common.cuh")
    (dst / "common.cuh").write_text(t)
    shutil.copy(cdir / "math.cuh", dst / "math.cuh")
    shutil.copy(cdir / "util.cuh", dst / "util.cuh")
    shutil.copy(cdir / "SPH" / "kernel.cuh", dst / "kernel.cuh")
    shutil.copy(cdir / "nsearch" / "morton.cuh", dst / "morton.cuh")


def variant_config(spec: dict) -> str:
    v = dict(REF_DEFAULT)
    v.update(spec)
    if isinstance(v["k"], tuple):
        v["k"] = textbook_stiffness(v["k"][1], v["r"])
    n, nb = v["n"], v["nb"]
    lines = [
        "#pragma once",
        f"#define REF_PARTICLE_RADIUS {v['r']!r}f",
        f"#define REF_STIFFNESS {v['k']:.9g}f",
        f"#define REF_VISCOSITY {v['nu']!r}f",
        f"#define REF_SURFACE_TENSION {v['alpha']!r}f",
        f"#define REF_GX {v['g'][0]!r}f",
        f"#define REF_GY {v['g'][1]!r}f",
        f"#define REF_GZ {v['g'][2]!r}f",
        f"#define REF_EXTERNAL_FORCE {v['force']}",
        f"#define REF_CELL_SIZE_MULT {v['cell_mult']}",
        f"#define REF_TABLE_SIZE_MULT {v['table_mult']}",
        f"#define REF_MIN_TABLE_SIZE {bit_ceil(n) // 4}",      # step_tuner.cuh:20
        f"#define REF_BOUNDARY_TABLE_SIZE {max(bit_ceil(nb) // 2, 1)}",  # rebuild_n_search.cuh:40-42
        f"#define REF_BLOCK {v['block']}",
        f"#define REF_FLUID_N {n}u",
        f"#define REF_BOUNDARY_N {nb}u",
        f"#define REF_MIN_TIME_STEP {v['min_dt']!r}f",
        f"#define REF_MAX_TIME_STEP {v['max_dt']!r}f",
        f"#define REF_CFL_FACTOR {v['cfl']!r}f",
        f"#define REF_NP_MAX_TIME_STEP {v['np_max']!r}f",
        "",
    ]
    return "\n".join(lines)


def nvcc(args, cwd):
    r = subprocess.run(["nvcc", *args], cwd=cwd, capture_output=True, text=True)
    if r.returncode != 0:
        raise SystemExit(f"nvcc failed: {' '.join(args)}\n{r.stdout}\n{r.stderr}")


def build_variant(ref: Path, name: str, spec: dict, jobs: int):
    vdir = OUT / name
    src = vdir / "src"
    shim_sources(ref, src)
    cfg = variant_config(spec)
    cfg_path = src / "variant_config.h"
    lib = vdir / "librefpath.so"
    stamp = vdir / "config.stamp"
    # rebuild when the variant's constants or the harness sources change
    import hashlib

    harness = b"".join((HERE / "refpath" / f).read_bytes() for f in ("refpath_host.cu", "ref_kernels.cu"))
    cfg_stamp = cfg + "// harness " + hashlib.sha256(harness).hexdigest() + "\n"
    if lib.exists() and stamp.exists() and stamp.read_text() == cfg_stamp:
        return name, "up to date"
    cfg_path.write_text(cfg)
    common = [*NVFLAGS, "-I", str(src), "-include", str(cfg_path)]
    objs = []
    jobs_list = []
    for fam, tag in FAMILIES.items():
        obj = vdir / f"fam_{tag}.o"
        objs.append(obj)
        jobs_list.append([*common, f"-DREF_FAMILY={fam}", f"-DREFNS=refns_{tag}", "-c", str(HERE / "refpath" / "ref_kernels.cu"), "-o",
                          str(obj)])
    host_obj = vdir / "refpath_host.o"
    objs.append(host_obj)
    jobs_list.append([*common, "-c", str(HERE / "refpath" / "refpath_host.cu"), "-o", str(host_obj)])
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        list(ex.map(lambda a: nvcc(a, vdir), jobs_list))
    nvcc([*ARCH, "-shared", "-o", str(lib), *map(str, objs), "-lcudart_static", "-lrt", "-ldl", "-lpthread"], vdir)
    stamp.write_text(cfg_stamp)
    return name, "built"


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("WCSPH_REFERENCE_DIR"),
                    help="checkout of petbab/fluid-simulation (or set WCSPH_REFERENCE_DIR)")
    ap.add_argument("--variants", nargs="*", default=list(VARIANTS))
    ap.add_argument("--jobs", type=int, default=max(os.cpu_count() or 4, 4))
    a = ap.parse_args()
    if not a.reference:
        print("build_ref: no reference checkout given (--reference or WCSPH_REFERENCE_DIR); skipping",
              file=sys.stderr)
        return
    ref = Path(a.reference)
    if not (ref / "src" / "cuda" / "tuning" / "kernels").is_dir():
        print(f"build_ref: no reference sources at {ref}; skipping", file=sys.stderr)
        return
    OUT.mkdir(exist_ok=True)
    for name in a.variants:
        print("build_ref:", *build_variant(ref, name, VARIANTS[name], a.jobs), flush=True)


if __name__ == "__main__":
    main()
