"""ORACLE -- test infrastructure only.

ctypes bridge to the CPU restatement of the reference (oracle/oracle.cpp,
built into oracle/_build/liboracle.so by oracle/build_oracle.py).  Only the
tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
use this package, as the checker; the product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

P, I, D = C.c_void_p, C.c_int, C.c_double
PI, PD = C.POINTER(C.c_int), C.POINTER(C.c_double)

_PROTO = {
    "orc_last_error": (C.c_char_p, []),
    "orc_set_threads": (None, [I]),
    "orc_get_threads": (I, []),
    "orc_mesh_create": (P, [I, PI, PD, D, D, I, PI, PI, PD]),
    "orc_mesh_destroy": (None, [P]),
    "orc_seeds_uniform": (None, [C.c_uint64, I, D, D, PD]),
    "orc_mesh_voronoi": (P, [PD, I, D, D, I, PI]),
    "orc_mesh_polys": (None, [P, PI, PD]),
    "orc_mesh_nnzb": (I, [P]),
    "orc_mesh_pattern": (None, [P, PI, PI]),
    "orc_mesh_nedges": (I, [P]),
    "orc_mesh_export": (None, [P, PI, PI, PD, PD, PD]),
    "orc_eq_create": (P, [P, I, I, D, D, D, I, PD, PD]),
    "orc_eq_destroy": (None, [P]),
    "orc_eq_set_exact_jacobian": (None, [P, I]),
    "orc_eq_nnzb": (I, [P]),
    "orc_assemble": (None, [P, PD, D, PD]),
    "orc_jacobian": (None, [P, PD, D, PI, PI, PD]),
    "orc_mass_blocks": (None, [P, PD]),
    "orc_mass_solve": (None, [P, PD, PD]),
    "orc_mass_matvec": (None, [P, PD, PD]),
    "orc_l2norm": (None, [P, PD, PD]),
    "orc_l2error": (None, [P, PD, I, PD, D, PD]),
    "orc_interp": (None, [P, I, PD, D, PD]),
    "orc_bsr_matvec": (None, [I, I, PI, PI, PD, PD, PD]),
    "orc_ilu0": (I, [I, I, PI, PI, PD, PD, PI, PI, PD, PI, PI, PD]),
    "orc_precond_apply": (None, [I, I, I, PI, PI, PD, PD]),
    "orc_gmres": (None, [I, I, I, PI, PI, PD, PD, PD, I, PD, PI]),
    "orc_jacobi": (None, [I, I, PI, PI, PD, PD, PD, PD, PI]),
    "orc_levels": (I, [I, PI, PI, PI, PI, PI, PI, PI]),
    "orc_stepper_create": (P, [P, I, I, I, D, I, D, I]),
    "orc_stepper_destroy": (None, [P]),
    "orc_step": (None, [P, PD, D, D, PI, PD]),
    "orc_leg2d": (D, [D, D, I, PD]),
    "orc_legder": (None, [I, PD, PD, PD]),
    "orc_tri_integral": (D, [PD, I, I, I]),
    "orc_line_integral": (D, [D, D, D, D, I, I, I]),
    "orc_gl_nodes": (None, [I, PD]),
}

_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            from .build_oracle import build
            build()
        lib = C.CDLL(LIB_PATH)
        for k, (r, a) in _PROTO.items():
            f = getattr(lib, k)
            f.restype = r
            f.argtypes = a
        _lib = lib
    return _lib


def pi(a):
    return a.ctypes.data_as(PI)


def pd(a):
    return a.ctypes.data_as(PD)


def i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def set_threads(n: int) -> None:
    load().orc_set_threads(n)


def get_threads() -> int:
    return load().orc_get_threads()


def uniform_seeds(seed: int, n: int, width: float = 1.0, height: float = 1.0) -> np.ndarray:
    """std::mt19937_64(seed): x = (g()>>11)*2^-53*width, then y."""
    xy = np.empty((n, 2))
    load().orc_seeds_uniform(C.c_uint64(seed), n, width, height, pd(xy))
    return xy


class Mesh:
    """Oracle mesh built from cell-frame polygons + sub-triangles."""

    @classmethod
    def voronoi(cls, seeds, width: float, height: float, periodic: bool = False, side_codes=None) -> "Mesh":
        """Brute-force (O(n^2)) Voronoi mesh of the seeds, built by the oracle
        alone; sub-triangles are the fans from the vertex centroids."""
        L = load()
        xy = f64(seeds)
        codes = None if side_codes is None else i32(side_codes)
        self = cls.__new__(cls)
        self.a = None
        self._keep = (xy, codes)
        self.n = len(xy)
        self.h = L.orc_mesh_voronoi(pd(xy), self.n, width, height, int(periodic),
                                    None if codes is None else pi(codes))
        return self

    def polygons(self):
        """(cell_ptr, poly_xy) in cell frames, after vertex deduplication"""
        L = load()
        E = L.orc_mesh_nedges(self.h)
        cp, xy = np.zeros(self.n + 1, np.int32), np.zeros((E, 2))
        L.orc_mesh_polys(self.h, pi(cp), pd(xy))
        return cp, xy

    def pattern(self):
        """Jacobian block pattern (rowptr, colidx) of the oracle's connectivity"""
        L = load()
        rp, cl = np.zeros(self.n + 1, np.int32), np.zeros(L.orc_mesh_nnzb(self.h), np.int32)
        L.orc_mesh_pattern(self.h, pi(rp), pi(cl))
        return rp, cl

    def __init__(self, arrays: dict, side_codes=None):
        L = load()
        self.a = arrays
        cp, xy = i32(arrays["cell_ptr"]), f64(arrays["poly_xy"])
        tp, tx = i32(arrays["tri_ptr"]), f64(arrays["tri_xy"])
        codes = None if side_codes is None else i32(side_codes)
        self._keep = (cp, xy, tp, tx, codes)
        self.n = len(cp) - 1
        self.h = L.orc_mesh_create(self.n, pi(cp), pd(xy), arrays["width"], arrays["height"],
                                   int(arrays["periodic"]), None if codes is None else pi(codes), pi(tp), pd(tx))

    def export(self):
        L = load()
        E = L.orc_mesh_nedges(self.h)
        cp = np.zeros(self.n + 1, np.int32)
        nbr = np.zeros(E, np.int32)
        sh = np.zeros((E, 2))
        bb = np.zeros((self.n, 4))
        nrm = np.zeros((E, 2))
        L.orc_mesh_export(self.h, pi(cp), pi(nbr), pd(sh), pd(bb), pd(nrm))
        return dict(cell_ptr=cp, edge_nbr=nbr, edge_shift=sh, bb=bb, normals=nrm)

    def __del__(self):
        try:
            load().orc_mesh_destroy(self.h)
        except Exception:
            pass


class Equation:
    ADV_CONST, ADV_ROT, EULER = 0, 1, 2

    def __init__(self, mesh: Mesh, physics: int, degree: int, gamma=1.4, beta=(1.0, 1.0), dkind=0, dparams=None,
                 inflow=None, exact_jacobian=False):
        L = load()
        self.mesh = mesh
        self.nc = 4 if physics == 2 else 1
        self.nb = (degree + 1) * (degree + 2) // 2
        self.bl = self.nb * self.nc
        self.n = mesh.n
        self.deg = degree
        dp = np.zeros(8)
        if dparams is not None:
            dp[: len(dparams)] = dparams
        inf = np.zeros(4)
        if inflow is not None:
            inf[: len(inflow)] = inflow
        self._keep = (dp, inf)
        self.h = L.orc_eq_create(mesh.h, physics, degree, gamma, beta[0], beta[1], dkind, pd(dp), pd(inf))
        if exact_jacobian:
            L.orc_eq_set_exact_jacobian(self.h, 1)

    @property
    def ndof(self):
        return self.n * self.bl

    def assemble(self, u, t=0.0):
        u = f64(u).ravel()
        b = np.zeros_like(u)
        load().orc_assemble(self.h, pd(u), t, pd(b))
        return b

    def jacobian(self, u, t=0.0):
        L = load()
        u = f64(u).ravel()
        nnzb = L.orc_eq_nnzb(self.h)
        rp = np.zeros(self.n + 1, np.int32)
        cl = np.zeros(nnzb, np.int32)
        bl = np.zeros((nnzb, self.bl, self.bl))
        L.orc_jacobian(self.h, pd(u), t, pi(rp), pi(cl), pd(bl))
        return rp, cl, bl

    def mass_blocks(self):
        out = np.zeros((self.n, self.bl, self.bl))
        load().orc_mass_blocks(self.h, pd(out))
        return out

    def mass_solve(self, x):
        x = f64(x).ravel()
        y = np.zeros_like(x)
        load().orc_mass_solve(self.h, pd(x), pd(y))
        return y

    def mass_matvec(self, x):
        x = f64(x).ravel()
        y = np.zeros_like(x)
        load().orc_mass_matvec(self.h, pd(x), pd(y))
        return y

    def l2norm(self, u):
        u = f64(u).ravel()
        out = np.zeros(4)
        load().orc_l2norm(self.h, pd(u), pd(out))
        return out[: self.nc]

    def l2error(self, u, kind, params, t=0.0):
        u = f64(u).ravel()
        p = np.zeros(8)
        p[: len(params)] = params
        out = np.zeros(4)
        load().orc_l2error(self.h, pd(u), kind, pd(p), t, pd(out))
        return out[: self.nc]

    def interp(self, kind, params, t=0.0):
        p = np.zeros(8)
        p[: len(params)] = params
        u = np.zeros(self.ndof)
        load().orc_interp(self.h, kind, pd(p), t, pd(u))
        return u

    def __del__(self):
        try:
            load().orc_eq_destroy(self.h)
        except Exception:
            pass


class Stepper:
    """kind / pc numbering as include/cpolyg.h (cpg_step_kind, cpg_pc_kind)."""

    def __init__(self, eq: Equation, kind: int, pc: int = 2, gmres_m=20, gmres_tol=1e-14, gmres_maxit=90000,
                 newton_tol=5e-13, newton_maxit=100):
        self.eq = eq
        self.h = load().orc_stepper_create(eq.h, kind, pc, gmres_m, gmres_tol, gmres_maxit, newton_tol,
                                           newton_maxit)
        self.stats = np.zeros(4, np.int32)
        self.res = np.zeros(1)

    def advance(self, u, dt, t=0.0):
        u = f64(u).ravel().copy()
        load().orc_step(self.h, pd(u), dt, t, pi(self.stats), pd(self.res))
        return u

    def __del__(self):
        try:
            load().orc_stepper_destroy(self.h)
        except Exception:
            pass


def bsr_matvec(rp, cl, blocks, x):
    rp, cl, blocks, x = i32(rp), i32(cl), f64(blocks), f64(x).ravel()
    y = np.zeros_like(x)
    load().orc_bsr_matvec(len(rp) - 1, blocks.shape[-1], pi(rp), pi(cl), pd(blocks), pd(x), pd(y))
    return y


def ilu0(rp, cl, blocks):
    """BlockILU0 factors: (DD[n], (Lrow, Lcol, L), (Urow, Ucol, DU), singular_row)"""
    rp, cl, blocks = i32(rp), i32(cl), f64(blocks)
    n, bl, nnzb = len(rp) - 1, blocks.shape[-1], len(cl)
    dd = np.zeros((n, bl, bl))
    lr, ur = np.zeros(n + 1, np.int32), np.zeros(n + 1, np.int32)
    lc, uc = np.zeros(max(nnzb, 1), np.int32), np.zeros(max(nnzb, 1), np.int32)
    lb, ub = np.zeros((max(nnzb, 1), bl, bl)), np.zeros((max(nnzb, 1), bl, bl))
    sing = load().orc_ilu0(n, bl, pi(rp), pi(cl), pd(blocks), pd(dd), pi(lr), pi(lc), pd(lb), pi(ur), pi(uc),
                           pd(ub))
    return dd, (lr, lc[: lr[-1]], lb[: lr[-1]]), (ur, uc[: ur[-1]], ub[: ur[-1]]), sing


def precond_apply(kind, rp, cl, blocks, x):
    rp, cl, blocks = i32(rp), i32(cl), f64(blocks)
    x = f64(x).ravel().copy()
    load().orc_precond_apply(kind, len(rp) - 1, blocks.shape[-1], pi(rp), pi(cl), pd(blocks), pd(x))
    return x


def gmres(pc_kind, rp, cl, blocks, b, x0, m, tol, maxit):
    rp, cl, blocks = i32(rp), i32(cl), f64(blocks)
    b = f64(b).ravel()
    x = f64(x0).ravel().copy()
    t = np.array([tol])
    mi = np.array([maxit], np.int32)
    load().orc_gmres(pc_kind, len(rp) - 1, blocks.shape[-1], pi(rp), pi(cl), pd(blocks), pd(b), pd(x), m, pd(t),
                     pi(mi))
    return x, int(mi[0]), float(t[0])


def jacobi(rp, cl, blocks, b, x0, tol, maxit):
    rp, cl, blocks = i32(rp), i32(cl), f64(blocks)
    b = f64(b).ravel()
    x = f64(x0).ravel().copy()
    t = np.array([tol])
    mi = np.array([maxit], np.int32)
    load().orc_jacobi(len(rp) - 1, blocks.shape[-1], pi(rp), pi(cl), pd(blocks), pd(b), pd(x), pd(t), pi(mi))
    return x, int(mi[0]), float(t[0])


def levels(rp, cl):
    rp, cl = i32(rp), i32(cl)
    n = len(rp) - 1
    nl = np.zeros(2, np.int32)
    lp, lr = np.zeros(n + 2, np.int32), np.zeros(n, np.int32)
    up, ur = np.zeros(n + 2, np.int32), np.zeros(n, np.int32)
    load().orc_levels(n, pi(rp), pi(cl), pi(lp), pi(lr), pi(up), pi(ur), pi(nl))
    return lp[: nl[0] + 1], lr, up[: nl[1] + 1], ur


def leg2d(x, y, m, c):
    c = f64(c)
    return load().orc_leg2d(x, y, m, pd(c))


def legder(m, c):
    c = f64(c)
    dx, dy = np.zeros(len(c)), np.zeros(len(c))
    load().orc_legder(m, pd(c), pd(dx), pd(dy))
    return dx, dy


def tri_integral(T, deg, a, b):
    T = f64(T)
    return load().orc_tri_integral(pd(T), deg, a, b)


def line_integral(x1, y1, x2, y2, deg, a, b):
    return load().orc_line_integral(x1, y1, x2, y2, deg, a, b)


def gl_nodes(m):
    out = np.zeros(m)
    load().orc_gl_nodes(m, pd(out))
    return out
