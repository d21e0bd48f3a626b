"""Generate the golden fixtures of tests/golden/ with the oracle.

Long oracle runs (tens of seconds to minutes of CPU) are recorded once here
and committed as small .npz files, so that the GPU tests compare the CUDA
path against the oracle's output without re-running the oracle on the GPU
host.  Each fixture stores the inputs that define the case (seeds, sizes,
time step), a digest of the mesh arrays it was computed on, the oracle's
final state and its per-step Newton/GMRES counts.

    python tests/golden/make_golden.py [case ...]

Cases:
  sdirk3_vortex_p3_1000 -- 2D Euler isentropic vortex (strength 5, centre
      (5,5), free stream (1,1), gamma 1.4) on the periodic [0,10]^2 with 1000
      Voronoi cells (seed 2), p=3, Alexander's L-stable SDIRK3 at the time
      step of the 100k-cell benchmark scaled by the cell size
      (dt = 0.05 * sqrt(100000/1000) = 0.5, the same dt/h), 20 steps,
      GMRES(30) + block ILU(0) tol 1e-10, Newton 5e-13, exact Jacobian.
"""
from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

VORTEX = [5.0, 5.0, 5.0, 1.0, 1.0, 1.4, 10.0, 10.0]
STEP_SDIRK3 = 10


def mesh_digest(arrays: dict) -> str:
    h = hashlib.sha256()
    for k in ("cell_ptr", "poly_xy", "edge_nbr", "edge_shift", "tri_ptr", "tri_xy"):
        h.update(np.ascontiguousarray(arrays[k]).tobytes())
    return h.hexdigest()


def sdirk3_vortex(n: int = 1000, degree: int = 3, steps: int = 20) -> dict:
    import cpolyg_b200 as cp  # host mesher only (no GPU needed)
    import oracle
    dt = 0.05 * (100000 / n) ** 0.5
    m = cp.PolyMesh.voronoi(cp.uniform_seeds(2, n, 10.0, 10.0), 10.0, 10.0, periodic=True)
    arrays = m.export()
    om = oracle.Mesh(arrays)
    oe = oracle.Equation(om, 2, degree, dkind=2, dparams=VORTEX, exact_jacobian=True)
    u0 = oe.interp(2, VORTEX)
    st = oracle.Stepper(oe, STEP_SDIRK3, pc=2, gmres_m=30, gmres_tol=1e-10, gmres_maxit=90000)
    u, t = u0.copy(), 0.0
    newton, gmres = [], []
    for k in range(steps):
        t0 = time.time()
        u = st.advance(u, dt, t)
        t += dt
        newton.append(int(st.stats[0]))
        gmres.append(int(st.stats[1]))
        print(f"  step {k + 1}: newton {newton[-1]} gmres {gmres[-1]} ({time.time() - t0:.1f} s)", flush=True)
        assert st.stats[3] == 1, "oracle Newton did not converge"
    return dict(n=n, degree=degree, seed=2, dt=dt, steps=steps, mesh_sha256=mesh_digest(arrays), u=u,
                newton=np.array(newton), gmres=np.array(gmres))


CASES = {"sdirk3_vortex_p3_1000": sdirk3_vortex}


def main(names):
    for name in names or CASES:
        print(name, flush=True)
        out = CASES[name]()
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)


if __name__ == "__main__":
    main(sys.argv[1:])
