"""The C++ interface (include/cpolyg.hpp) as a drop-in for the reference's
driver code: tests/cpp/drop_in_rk4.cpp is written the way the reference's
examples use PolyMesh / Equation / TimeStepper.  It must compile against the
headers and link the shared library with a plain g++ (CPU test), and on a GPU
its result must equal the Python path's bit for bit (same kernels, same
launch sequence)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "cpolyg_b200", "_lib")


def build_dropin(tmp_path) -> str:
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    if not os.path.exists(os.path.join(LIBDIR, "libcpolyg_b200.so")):
        from cpolyg_b200 import build
        build.build()
    cuda = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    exe = str(tmp_path / "drop_in_rk4")
    cmd = [gxx, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"), "-I", os.path.join(cuda, "include"),
           os.path.join(ROOT, "tests", "cpp", "drop_in_rk4.cpp"), "-L", LIBDIR, "-lcpolyg_b200",
           "-L", os.path.join(cuda, "lib64"), "-lcudart", f"-Wl,-rpath,{LIBDIR}",
           f"-Wl,-rpath,{os.path.join(cuda, 'lib64')}", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return exe


def test_cpp_interface_compiles_and_links(tmp_path):
    exe = build_dropin(tmp_path)
    assert os.access(exe, os.X_OK)


@pytest.mark.gpu
def test_cpp_rk4_matches_python_path_bitwise(tmp_path, ctx):
    import cpolyg_b200 as cp
    exe = build_dropin(tmp_path)
    r = subprocess.run([exe, "1000", "10"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    l2 = None
    coef = {}
    for ln in r.stdout.splitlines():
        f = ln.split()
        if f[0] == "l2":
            l2 = float(f[1])
        elif f[0] == "u":
            coef[int(f[1])] = float(f[2])
    mesh = cp.PolyMesh.voronoi(cp.uniform_seeds(1, 1000, 1.0, 1.0), 1.0, 1.0, periodic=True)
    eq = cp.ConstantAdvection(ctx, mesh, 2, 1.0, 1.0)
    u = eq.interp(cp.INIT_GAUSSIAN, [100.0, 0.5, 0.5])
    st = cp.RK4(eq)
    t, dt = 0.0, 1e-4
    for _ in range(10):
        st.advance(u, dt, t)
        t += dt
    h = u.cpu().numpy().ravel()
    assert np.array_equal(h[:6], np.array([coef[i] for i in range(6)]))
    assert float(eq.L2Norm(u)[0]) == l2
