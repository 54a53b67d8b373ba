"""Builds the engine library in-tree: sphere_b200/libsphere_b200.so.

Every CUDA source is compiled for sm_100a only.  The FP64 DEM kernels are
compiled with -fmad=false so their arithmetic rounds like the reference's
--fmad=false build.
"""
from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libsphere_b200.so")
BUILD = os.path.join(HERE, "_build")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]
# kernels whose results must round exactly like the reference
NO_FMA = {"dem_kernels.cu", "sort.cu", "darcy.cu", "persistent_fp64.cu", "stats.cu", "render.cu",
          "navierstokes.cu"}
SOURCES = ["bin_io.cpp", "dem_kernels.cu", "sort.cu", "engine.cu", "darcy.cu", "dem_mixed.cu",
           "noalloc_sort.cu", "engine_persist.cu", "persistent_fp64.cu", "persistent_mixed.cu",
           "batch.cu", "warmstart.cu", "stats.cu", "render.cu", "navierstokes.cu"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _needs(obj: str, deps) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, ptxas_info: bool = False, out: str = OUT,
          build_dir: str = BUILD, defines=()) -> str:
    os.makedirs(build_dir, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "sphere_b200.h"))
    objs = []
    nv = nvcc()
    jobs = []
    for src in SOURCES:
        path = os.path.join(CSRC, src)
        obj = os.path.join(build_dir, src + ".o")
        objs.append(obj)
        if not _needs(obj, [path, __file__] + headers):
            continue
        cmd = [nv] + COMMON + ARCH + ["-c", path, "-o", obj]
        if src.endswith(".cpp"):
            cmd = [nv, "-x", "c++"] + COMMON + ["-c", path, "-o", obj]
        if src in NO_FMA:
            cmd.insert(1, "-fmad=false")
        cmd += [f"-D{d}" for d in defines]
        if ptxas_info and src.endswith(".cu"):
            cmd += ["-Xptxas", "-v"]
        if verbose:
            print(" ".join(cmd), flush=True)
        jobs.append(cmd)
    # translation units compile independently
    with concurrent.futures.ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as ex:
        for f in [ex.submit(subprocess.check_call, c) for c in jobs]:
            f.result()
    if _needs(out, objs):
        cmd = [nv, "-shared"] + ARCH + ["-o", out] + objs + ["-lcuda"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
    return out


if __name__ == "__main__":
    build(verbose=True, ptxas_info="-v" in sys.argv)
