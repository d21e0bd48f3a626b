"""Shared test cases: seeded meshes and the matching oracle objects."""
from __future__ import annotations

import functools

import numpy as np

import cpolyg_b200 as cp
import oracle

GAMMA = 1.4


@functools.lru_cache(maxsize=None)
def mesh(n: int, periodic: bool, width: float = 1.0, seed: int = 1, codes: tuple | None = None):
    seeds = cp.uniform_seeds(seed, n, width, width)
    m = cp.PolyMesh.voronoi(seeds, width, width, periodic=periodic, side_codes=None if codes is None else list(codes))
    arrays = m.export()
    om = oracle.Mesh(arrays, side_codes=None if codes is None else list(codes))
    return m, arrays, om


def vortex_params(width: float, strength: float = 5.0):
    c = width / 2
    return [strength, c, c, 1.0, 1.0, GAMMA, width, width]


# (physics, degree, kwargs for both sides, init kind, init params builder)
PHYSICS = {
    "adv_const": dict(phys=cp.ADVECTION_CONST, beta=(1.0, 1.0)),
    "adv_rot": dict(phys=cp.ADVECTION_ROTATING, beta=(0.0, 0.0)),
    "euler": dict(phys=cp.EULER, beta=(0.0, 0.0)),
}


def init_field(phys: int, width: float):
    if phys == cp.EULER:
        return cp.INIT_VORTEX, vortex_params(width)
    return cp.INIT_GAUSSIAN, [100.0 / width ** 2, 0.5 * width, 0.5 * width]


def equations(ctx, name: str, degree: int, n: int = 300, periodic: bool = True, width: float = 1.0,
              codes: tuple | None = None, dirichlet=None, inflow=None, exact_jacobian: bool = False,
              oracle_exact: bool | None = None):
    """(gpu Equation, oracle Equation, mesh arrays)"""
    m, arrays, om = mesh(n, periodic, width, 1, codes)
    p = PHYSICS[name]
    dk, dp = dirichlet if dirichlet is not None else init_field(p["phys"], width)
    ge = cp.Equation(ctx, m, p["phys"], degree, gamma=GAMMA, beta=p["beta"], dirichlet=(dk, dp), inflow=inflow,
                     exact_jacobian=exact_jacobian)
    oe = oracle.Equation(om, p["phys"], degree, gamma=GAMMA, beta=p["beta"], dkind=dk, dparams=dp, inflow=inflow,
                         exact_jacobian=exact_jacobian if oracle_exact is None else oracle_exact)
    return ge, oe, arrays


def rel(a, b) -> float:
    a = np.asarray(a, dtype=np.float64).ravel()
    b = np.asarray(b, dtype=np.float64).ravel()
    d = np.abs(a - b).max() if a.size else 0.0
    s = max(np.abs(b).max() if b.size else 0.0, 1e-300)
    return float(d / s)


def to_np(t) -> np.ndarray:
    return t.detach().cpu().numpy().ravel()


def to_dev(a, like=None):
    import torch
    t = torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64)).cuda()
    if like is not None:
        t = t.reshape(like.shape)
    return t.contiguous()
