"""Build recipe of the oracle (test infrastructure only).

* ``oracle/_build/liboracle.so`` from ``oracle/oracle.cpp`` (the CPU
  restatement of the reference, OpenMP over cells), always.
* ``oracle/_ref/`` from the reference's own sources, only when they are
  present (``CPOLYG_REFERENCE_SRC``, by default ``/root/reference``): the
  vendored Triangle and Voro++ 2D
  libraries, compiled unmodified where they lie, plus the small driver
  ``oracle/ref_mesh_driver.cpp`` that calls them the way
  ``PolyMesh(pts, w, h)`` and ``Triangulation`` do (src/PolyMesh.cpp:162-218,
  src/Triangulation.cpp:11-101).  The rest of the reference needs Armadillo,
  GSL and LAPACK, which are not available, so it is not built.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
REF_OUT = os.path.join(HERE, "_ref")
# the reference's source tree (read only); CPOLYG_REFERENCE_SRC overrides it
REF_SRC = os.environ.get("CPOLYG_REFERENCE_SRC", "/root/reference")

CXXFLAGS = ["-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fopenmp", "-fPIC", "-std=c++17"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)


def build_oracle() -> str:
    os.makedirs(BUILD, exist_ok=True)
    src = os.path.join(HERE, "oracle.cpp")
    out = os.path.join(BUILD, "liboracle.so")
    if not os.path.exists(out) or os.path.getmtime(out) < os.path.getmtime(src):
        _run(["g++", *CXXFLAGS, "-shared", "-o", out, src])
    return out


def build_ref() -> str | None:
    """Compile the reference's Triangle + Voro++ into oracle/_ref (if present)."""
    tri = os.path.join(REF_SRC, "src", "triangle", "triangle.c")
    vsrc = os.path.join(REF_SRC, "voro++_2d", "src")
    driver = os.path.join(HERE, "ref_mesh_driver.cpp")
    if not (os.path.exists(tri) and os.path.isdir(vsrc) and os.path.exists(driver)):
        return None
    os.makedirs(REF_OUT, exist_ok=True)
    out = os.path.join(REF_OUT, "libref_mesh.so")
    if os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(driver):
        return out
    tri_o = os.path.join(REF_OUT, "triangle.o")
    # Triangle: the file configures itself as a double-precision library
    # (src/triangle/triangle.c:213-219)
    _run(["gcc", "-O2", "-fPIC", "-DNO_TIMER", "-w", "-c", tri, "-o", tri_o])
    # Voro++ 2D: the single amalgamated translation unit of the library
    voro_o = os.path.join(REF_OUT, "voro2d.o")
    _run(["g++", "-O2", "-fPIC", "-w", "-I", vsrc, "-c", os.path.join(vsrc, "voro++_2d.cc"), "-o", voro_o])
    _run(["g++", "-O2", "-fPIC", "-shared", "-std=c++17", "-I", vsrc, "-I", os.path.join(REF_SRC, "src", "triangle"),
          "-o", out, driver, tri_o, voro_o])
    return out


def build() -> None:
    build_oracle()
    try:
        build_ref()
    except RuntimeError as e:  # the pins are optional; the oracle itself is not
        sys.stderr.write(str(e) + "\n")


if __name__ == "__main__":
    build()
    print("oracle built:", build_oracle(), "ref:", build_ref())
