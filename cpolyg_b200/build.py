"""In-tree build of libcpolyg_b200.so (sm_100a CUDA kernels + C ABI).

Run ``python -m cpolyg_b200.build`` (or ``__graft_entry__.build()``).  The
shared library lands in ``cpolyg_b200/_lib/`` and object files in
``cpolyg_b200/_build/``; nothing is installed elsewhere.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libcpolyg_b200.so")

CU_SOURCES = ["core.cu", "equation.cu", "bsr.cu", "precond.cu", "krylov.cu", "stepper.cu", "output.cu"]
CXX_SOURCES = ["mesh.cpp"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-Xptxas", "-warn-spills"]
CXX_FLAGS = ["-O2", "-std=c++17", "-fPIC", "-Wall"]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build step failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
    if r.stderr.strip():
        sys.stderr.write(r.stderr)


def _stale(out: str, deps: list[str]) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose: bool = False, jobs: int | None = None) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    nvcc = _nvcc()
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".hpp", ".h"))]
    headers.append(os.path.join(os.path.dirname(HERE), "include", "cpolyg.h"))
    steps = []
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _stale(o, [s] + headers):
            steps.append([nvcc, *ARCH, *NVCC_FLAGS, "-c", s, "-o", o])
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if _stale(o, [s] + headers):
            steps.append(["g++", *CXX_FLAGS, "-c", s, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        for f in [ex.submit(_run, c) for c in steps]:
            f.result()
    if steps or _stale(LIB, objs):
        _run([nvcc, *ARCH, "-shared", "-o", LIB, *objs, "-lcudart_static", "-lrt", "-ldl", "-lpthread"])
    if verbose:
        print("built", LIB)
    return LIB


if __name__ == "__main__":
    build(verbose=True)
