"""Builds the CUDA engine (sm_100a) into gpp_b200/libgpp_b200.so with nvcc.

Usage: python build.py [-j N]
Every translation unit is compiled with -gencode arch=compute_100a,code=sm_100a
and --fmad=false (so FP64 results are reproducible against the CPU restatement
used by the tests), then linked into one shared library exporting the C ABI
of include/gpp.h.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "gpp_b200", "libgpp_b200.so")
OBJ = os.path.join(HERE, "_build")
NVCC = os.environ.get("NVCC", "nvcc")
FLAGS = ["-std=c++17", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "--fmad=false",
         "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden", "--expt-relaxed-constexpr",
         "--extended-lambda", "-I", os.path.join(HERE, "..", "include")]
UNITS = ["common.cu", "live.cu", "compact.cu", "recovery.cu", "rules_cleanup.cu", "rules_bound.cu", "rules_propagation.cu", "sort.cu", "sort_static.cu", "rules_parallel.cu", "rules_singleton.cu", "rules_doubleton.cu", "rules_startup.cu", "rules_pwl_abs.cu", "rules_pwl_pair.cu",
         "engine.cu", "postsolve.cu", "folding.cu", "schedule_mlp.cu", "mps_reader.cpp", "capi.cu"]


def _compile(unit: str) -> str:
    src = os.path.join(SRC, unit)
    obj = os.path.join(OBJ, unit + ".o")
    deps = [src] + [os.path.join(SRC, f) for f in os.listdir(SRC) if f.endswith((".cuh", ".hpp"))]
    deps.append(os.path.join(HERE, "..", "include", "gpp.h"))
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps):
        return obj
    cmd = [NVCC, *FLAGS, "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {unit}:\n{r.stderr}")
    return obj


def build(jobs: int = 8) -> str:
    os.makedirs(OBJ, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(_compile, UNITS))
    if os.path.exists(OUT) and os.path.getmtime(OUT) >= max(os.path.getmtime(o) for o in objs):
        return OUT
    cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs, "-o", OUT]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stderr}")
    return OUT


if __name__ == "__main__":
    jobs = int(sys.argv[sys.argv.index("-j") + 1]) if "-j" in sys.argv else 8
    print(build(jobs))
