"""Build libcudasph_b200.so (sm_100a) in-tree with nvcc.

Usage: ``python -m cudasph_b200.build`` (or ``__graft_entry__.build()``).
The library lands in ``cudasph_b200/_lib/``; object files in
``cudasph_b200/_build/``.  The translation unit of the FP64 h solve and
neighbour predicate is compiled with ``-fmad=false`` so it performs the same
IEEE operations as an FP64 CPU evaluation.
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
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libcudasph_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
          "-I" + os.path.join(HERE, "..", "include")]
# no FMA contraction: the h solve's ranges and neighbour sets reproduce an FP64
# CPU evaluation bit for bit
NO_FMAD = {"neighbours.cu"}
SOURCES = ["sort.cu", "tree.cu", "neighbours.cu", "hydro.cu", "hydro_mixed.cu", "gravity.cu", "integrate.cu",
           "capi.cu", "legacy.cu", "peak.cu", "adjoint.cu", "treegrav.cu"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _compile(src: str, verbose_ptxas: bool) -> str:
    obj = os.path.join(BUILD, src.replace(".cu", ".o"))
    path = os.path.join(CSRC, src)
    deps = [path] + [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith(".cuh")]
    deps.append(os.path.join(HERE, "..", "include", "cudasph_b200.h"))
    if os.path.exists(obj) and not verbose_ptxas and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps):
        return obj
    cmd = [nvcc()] + ARCH + COMMON + ["-c", path, "-o", obj]
    if src in NO_FMAD:
        cmd.insert(1, "-fmad=false")
    if verbose_ptxas:
        cmd += ["-Xptxas", "-v"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose_ptxas:
        sys.stderr.write(r.stderr)
    return obj


def build_library(verbose_ptxas: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose_ptxas), SOURCES))
    if os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(o) for o in objs):
        return LIB
    cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build_library(verbose_ptxas="-v" in sys.argv))
