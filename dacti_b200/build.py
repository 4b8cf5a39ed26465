"""Builds the CUDA library ``dacti_b200/libdacti_gpu.so`` for sm_100a with nvcc.

Every translation unit is compiled with ``--fmad=false``: the FP64 solver keeps the reference's
operation order and rounding (no fused multiply-add contraction), which is what makes it
bit-compatible with the reference CPU solver.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libdacti_gpu.so")

UNITS = ["capi.cu", "noalloc.cu", "forecast.cu", "scene_build.cu", "solver_euler.cu", "solver_ns.cu", "solver_multi.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "--fmad=false", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "--expt-relaxed-constexpr", "-I" + os.path.join(HERE, "..", "include")]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _sources_newer_than(target: str) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    for root, _, files in os.walk(CSRC):
        for f in files:
            if os.path.getmtime(os.path.join(root, f)) > t:
                return True
    hdr = os.path.join(HERE, "..", "include", "dacti_gpu.h")
    return os.path.getmtime(hdr) > t


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    if not force and not _sources_newer_than(LIB):
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    cc = nvcc()
    extra = ["-Xptxas", "-v"] if ptxas_info else []

    def compile_one(unit: str) -> str:
        obj = os.path.join(BUILD, unit.replace(".cu", ".o"))
        cmd = [cc, *ARCH, *FLAGS, *extra, "-c", os.path.join(CSRC, unit), "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {unit}:\n{r.stderr[-6000:]}")
        if verbose or ptxas_info:
            sys.stderr.write(r.stderr)
        return obj

    with ThreadPoolExecutor(max_workers=len(UNITS)) as ex:
        objs = list(ex.map(compile_one, UNITS))
    tmp = LIB + ".tmp"
    # the library carries its own (static) CUDA runtime, independent of any runtime a host process
    # such as torch loads
    cmd = [cc, *ARCH, "-shared", "-cudart", "static", "-o", tmp, *objs]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr[-4000:]}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True, ptxas_info="--ptxas" in sys.argv)
    print(LIB)
