"""Builds the in-tree CUDA library ``asgard_b200/libasgard_b200.so`` for sm_100a.

    python asgard_b200/build.py

Each source is compiled by nvcc (``-gencode arch=compute_100a,code=sm_100a
-lineinfo -O3``) in parallel, then linked into one shared library exporting
the C ABI of ``include/asgard_b200.h``.  Objects go to ``_build/``.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(HERE, "libasgard_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise FileNotFoundError("nvcc not found")
    return cand


def _host_cxx() -> str:
    # the system g++ links the OpenMP runtime used by the grid builder
    return "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"


def sources():
    out = []
    for f in sorted(os.listdir(CSRC)):
        if f.endswith((".cu", ".cpp")):
            out.append(os.path.join(CSRC, f))
    return out


def _compile(src: str, verbose_ptxas: bool) -> str:
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    deps = [src] + [os.path.join(CSRC, h) for h in os.listdir(CSRC)
                    if h.endswith((".cuh", ".h"))] + [os.path.join(INCLUDE, "asgard_b200.h")]
    if os.path.exists(obj) and all(os.path.getmtime(obj) >= os.path.getmtime(d) for d in deps):
        return obj
    cmd = [_nvcc(), "-ccbin", _host_cxx(), "-std=c++17", "-O3", "-lineinfo",
           *ARCH, "-Xcompiler", "-fPIC,-fopenmp", "-I", INCLUDE, "-I", CSRC,
           "--expt-relaxed-constexpr", "-c", src, "-o", obj]
    if verbose_ptxas and src.endswith(".cu"):
        cmd.insert(1, "-Xptxas=-v")
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if verbose_ptxas:
        sys.stderr.write(r.stderr)
    return obj


def build(verbose_ptxas: bool = False, jobs: int | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose_ptxas), srcs))
    if not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [_nvcc(), "-ccbin", _host_cxx(), *ARCH, "-shared", "-o", LIB,
               *objs, "-Xcompiler", "-fopenmp", "-lgomp", "-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return LIB


if __name__ == "__main__":
    print(build(verbose_ptxas="-v" in sys.argv))
