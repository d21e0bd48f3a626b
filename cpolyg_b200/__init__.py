"""cpolyg_b200: B200 (sm_100a) implementation of cpolyg's polygonal DG hot path.

Python mirror of the reference's C++ interface (same class and method names as
src/PolyMesh.h, src/Equation.h, src/MassMatrix.h, src/BlockMatrix.h,
src/Jacobian.h, src/Preconditioners.h, src/TimeIntegration.h), calling the
library's C ABI (include/cpolyg.h) through ctypes.  Fields (MeshFn) are
float64 CUDA tensors of shape (n_cells, nc, nb), whose flat order is the
reference's arma::cube(nb, nc, n) order.  Device memory and streams come from
PyTorch; all arithmetic runs in the library's CUDA kernels.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _capi
from ._capi import (ADVECTION_CONST, ADVECTION_ROTATING, BC_DIRICHLET, BC_INFLOW, BC_OUTFLOW, BC_WALL, EULER, F32,
                    F64, INIT_CONSTANT, INIT_DENSITY_BUMP, INIT_GAUSSIAN, INIT_VORTEX, PC_BJACOBI, PC_ILU0, PC_NONE,
                    PC_STAGE_BJACOBI, STEP_BACKWARD_EULER, STEP_DIRK3, STEP_DIRK5, STEP_FORWARD_EULER, STEP_IRK2,
                    STEP_IRK2_INV, STEP_IRK3, STEP_IRK3_INV, STEP_RK2, STEP_RK4, STEP_SDIRK3, CpgError)

__all__ = [
    "lib", "Context", "PolyMesh", "Equation", "Advection", "ConstantAdvection", "Euler", "BlockMatrix",
    "Jacobian", "NoPreconditioner", "BlockJacobi", "BlockILU0", "TimeStepper", "ForwardEuler", "RK2", "RK4",
    "BackwardEuler", "DIRK", "SDIRK3", "IRK", "CpgError",
]


def lib() -> C.CDLL:
    return _capi.load()


def _pi(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_int))


def _pd(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _ptr(t) -> int:
    """device pointer of a float64 CUDA tensor (contiguous)"""
    import torch
    if not (isinstance(t, torch.Tensor) and t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
        raise TypeError("expected a contiguous float64 CUDA tensor")
    return t.data_ptr()


class Context:
    """Device + stream owning all library calls (cpg_ctx)."""

    def __init__(self, device: int = 0, stream=None):
        import torch
        self._lib = lib()
        if stream is None:
            stream = torch.cuda.current_stream(device)
        self.device = device
        self.stream = stream
        h = C.c_void_p()
        self._check(self._lib.cpg_ctx_create(device, C.c_void_p(stream.cuda_stream), C.byref(h)), None)
        self.h = h

    def _check(self, status: int, h=None) -> None:
        if status != 0:
            msg = self._lib.cpg_last_error(h if h is not None else getattr(self, "h", None))
            raise CpgError(status, msg.decode() if msg else "")

    def check(self, status: int) -> None:
        self._check(status, self.h)

    def sync(self) -> None:
        self.check(self._lib.cpg_ctx_sync(self.h))

    @property
    def launches(self) -> int:
        return int(self._lib.cpg_ctx_launch_count(self.h))

    def close(self) -> None:
        if getattr(self, "h", None):
            self._lib.cpg_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def uniform_seeds(seed: int, n: int, width: float = 1.0, height: float = 1.0) -> np.ndarray:
    """Seeds of std::mt19937_64(seed): x = (g()>>11)*2^-53*width, then y."""
    xy = np.empty((n, 2), dtype=np.float64)
    st = lib().cpg_seeds_uniform(C.c_uint64(seed), n, width, height, _pd(xy))
    if st != 0:
        raise CpgError(st, "seeds")
    return xy


class PolyMesh:
    """Host polygonal mesh (PolyMesh, src/PolyMesh.h:13-55)."""

    def __init__(self, handle, keep=None):
        self._lib = lib()
        self.h = handle
        info = _capi.MeshInfo()
        self._lib.cpg_mesh_get_info(self.h, C.byref(info))
        self.np = info.n_cells
        self.n_verts = info.n_verts
        self.n_edges = info.n_edges
        self.n_tris = info.n_tris
        self.periodic = bool(info.periodic)
        self.width, self.height = info.width, info.height

    @classmethod
    def voronoi(cls, seeds: np.ndarray, width: float = 1.0, height: float = 1.0, periodic: bool = False,
                side_codes=None) -> "PolyMesh":
        seeds = np.ascontiguousarray(seeds, dtype=np.float64)
        h = C.c_void_p()
        codes = None if side_codes is None else np.ascontiguousarray(side_codes, dtype=np.int32)
        st = lib().cpg_mesh_voronoi(_pd(seeds), len(seeds), width, height, int(periodic),
                                    None if codes is None else _pi(codes), C.byref(h))
        if st != 0:
            raise CpgError(st, "Voronoi mesh construction failed")
        return cls(h)

    @classmethod
    def from_polygons(cls, polys, width: float, height: float, periodic: bool = False,
                      side_codes=None) -> "PolyMesh":
        ptr = np.zeros(len(polys) + 1, dtype=np.int32)
        for i, p in enumerate(polys):
            ptr[i + 1] = ptr[i] + len(p)
        xy = np.ascontiguousarray(np.concatenate([np.asarray(p, dtype=np.float64) for p in polys]))
        codes = None if side_codes is None else np.ascontiguousarray(side_codes, dtype=np.int32)
        h = C.c_void_p()
        st = lib().cpg_mesh_from_polygons(len(polys), _pi(ptr), _pd(xy), width, height, int(periodic),
                                          None if codes is None else _pi(codes), C.byref(h))
        if st != 0:
            raise CpgError(st, "mesh construction failed")
        return cls(h)

    def set_subtriangles(self, tri_ptr, tri_xy) -> None:
        """Volume quadrature on these triangles (cell frame, 6 numbers each)
        instead of the centroid fans, e.g. the reference's Triangle "zQq"
        sub-triangulation; equations created afterwards use them."""
        tp = np.ascontiguousarray(tri_ptr, dtype=np.int32)
        tx = np.ascontiguousarray(tri_xy, dtype=np.float64).reshape(-1, 6)
        if len(tp) != self.np + 1 or tp[-1] != len(tx):
            raise ValueError("tri_ptr must have n_cells + 1 entries ending at the triangle count")
        st = self._lib.cpg_mesh_set_subtriangles(self.h, _pi(tp), _pd(tx))
        if st != 0:
            raise CpgError(st, "sub-triangles do not tile the cells")
        info = _capi.MeshInfo()
        self._lib.cpg_mesh_get_info(self.h, C.byref(info))
        self.n_tris = info.n_tris

    def gnuplot(self, path: str = "plt/edges.gnu") -> None:
        """PolyMesh::gnuplot: polygon outlines as gnuplot text."""
        st = self._lib.cpg_mesh_write_gnuplot(self.h, str(path).encode())
        if st != 0:
            raise CpgError(st, f"cannot write {path}")

    def export(self) -> dict:
        n, E, T = self.np, self.n_edges, self.n_tris
        out = dict(cell_ptr=np.zeros(n + 1, np.int32), poly_xy=np.zeros((E, 2)), vert_id=np.zeros(E, np.int32),
                   edge_nbr=np.zeros(E, np.int32), edge_shift=np.zeros((E, 2)), bb=np.zeros((n, 4)),
                   tri_ptr=np.zeros(n + 1, np.int32), tri_xy=np.zeros((T, 6)))
        self._lib.cpg_mesh_export(self.h, _pi(out["cell_ptr"]), _pd(out["poly_xy"]), _pi(out["vert_id"]),
                                  _pi(out["edge_nbr"]), _pd(out["edge_shift"]), _pd(out["bb"]),
                                  _pi(out["tri_ptr"]), _pd(out["tri_xy"]))
        out.update(width=self.width, height=self.height, periodic=self.periodic)
        return out

    def pattern(self):
        """Jacobian block pattern (rowptr, colidx), computed on the host."""
        nnzb = C.c_int64()
        rp = np.zeros(self.np + 1, np.int32)
        self._lib.cpg_mesh_pattern(self.h, _pi(rp), None, C.byref(nnzb))
        cl = np.zeros(nnzb.value, np.int32)
        self._lib.cpg_mesh_pattern(self.h, _pi(rp), _pi(cl), C.byref(nnzb))
        return rp, cl

    def __del__(self):
        try:
            if self.h:
                self._lib.cpg_mesh_destroy(self.h)
                self.h = None
        except Exception:
            pass


def pattern_levels(rowptr: np.ndarray, colidx: np.ndarray):
    """ILU(0) level schedule of a block pattern (host)."""
    rowptr = np.ascontiguousarray(rowptr, np.int32)
    colidx = np.ascontiguousarray(colidx, np.int32)
    n = len(rowptr) - 1
    nl, nu = C.c_int(), C.c_int()
    L = lib()
    L.cpg_pattern_levels(n, _pi(rowptr), _pi(colidx), C.byref(nl), None, None, C.byref(nu), None, None)
    lp, lr = np.zeros(nl.value + 1, np.int32), np.zeros(n, np.int32)
    up, ur = np.zeros(nu.value + 1, np.int32), np.zeros(n, np.int32)
    L.cpg_pattern_levels(n, _pi(rowptr), _pi(colidx), C.byref(nl), _pi(lp), _pi(lr), C.byref(nu), _pi(up),
                         _pi(ur))
    return lp, lr, up, ur


@dataclass
class Physics:
    kind: int
    gamma: float = 1.4
    beta: tuple = (1.0, 1.0)


class Equation:
    """Equation (src/Equation.h): residual, Jacobian, mass matrix, norms."""

    def __init__(self, ctx: Context, msh: PolyMesh, physics: int, degree: int, gamma: float = 1.4,
                 beta=(1.0, 1.0), dirichlet=(INIT_CONSTANT, None), inflow=None, exact_jacobian: bool = False):
        """exact_jacobian=False keeps the reference's Euler Jacobian (an inexact
        A_x entry and own-state neighbour blocks); True uses exact derivatives
        (same residual and converged solution, quadratic Newton)."""
        self.ctx = ctx
        self.msh = msh
        self._lib = ctx._lib
        d = _capi.EquationDesc()
        d.physics = physics
        d.degree = degree
        d.gamma = gamma
        d.exact_jacobian = int(exact_jacobian)
        d.beta[0], d.beta[1] = beta
        d.dirichlet_kind = dirichlet[0]
        for q, v in enumerate(dirichlet[1] or []):
            d.dirichlet_params[q] = v
        for q, v in enumerate(inflow or []):
            d.inflow_state[q] = v
        h = C.c_void_p()
        ctx.check(self._lib.cpg_equation_create(ctx.h, msh.h, C.byref(d), C.byref(h)))
        self.h = h
        info = _capi.EquationInfo()
        self._lib.cpg_equation_get_info(self.h, C.byref(info))
        self.info = info
        self.nb, self.nc, self.bl, self.np = info.nb, info.nc, info.bl, info.n_cells
        self.deg = degree
        self.physics = physics

    # MeshFn allocation
    def zeros(self):
        import torch
        return torch.zeros((self.np, self.nc, self.nb), dtype=torch.float64, device=f"cuda:{self.ctx.device}")

    def interp(self, kind: int, params, t: float = 0.0):
        """MeshFn::interp of an analytic field (cpg_init_kind)."""
        u = self.zeros()
        p = np.zeros(8)
        p[: len(params)] = params
        self.ctx.check(self._lib.cpg_interp(self.ctx.h, self.h, kind, _pd(p), t, C.c_void_p(_ptr(u))))
        return u

    def assemble(self, u, t: float = 0.0):
        b = self.zeros()
        self.ctx.check(self._lib.cpg_assemble(self.ctx.h, self.h, C.c_void_p(_ptr(u)), t, C.c_void_p(_ptr(b))))
        return b

    def jacobian(self, u, t: float = 0.0, scale: float = 1.0, add_mass: bool = False, precision: int = F64,
                 out: "BlockMatrix | None" = None) -> "Jacobian":
        J = out or Jacobian.for_equation(self, precision)
        self.ctx.check(self._lib.cpg_jacobian(self.ctx.h, self.h, C.c_void_p(_ptr(u)), t, scale, int(add_mass),
                                              J.h))
        return J

    # MassMatrix (src/MassMatrix.h)
    def mass_matvec(self, x):
        y = self.zeros()
        self.ctx.check(self._lib.cpg_mass_apply(self.ctx.h, self.h, C.c_void_p(_ptr(x)), C.c_void_p(_ptr(y))))
        return y

    def mass_solve(self, x):
        y = self.zeros()
        self.ctx.check(self._lib.cpg_mass_solve(self.ctx.h, self.h, C.c_void_p(_ptr(x)), C.c_void_p(_ptr(y))))
        return y

    def mass_blocks(self) -> np.ndarray:
        out = np.zeros((self.np, self.nb, self.nb))
        self.ctx.check(self._lib.cpg_mass_export(self.ctx.h, self.h, _pd(out)))
        return out  # [cell][j][k] = M(k, j)

    def L2Norm(self, u) -> np.ndarray:
        out = np.zeros(4)
        self.ctx.check(self._lib.cpg_l2norm(self.ctx.h, self.h, C.c_void_p(_ptr(u)), _pd(out)))
        return out[: self.nc].copy()

    def gnuplot(self, u, path: str) -> None:
        """MeshFn::gnuplot: field values at the 3-point rule of every
        sub-triangle, as gnuplot text."""
        self.ctx.check(self._lib.cpg_field_write_gnuplot(self.ctx.h, self.h, self.msh.h, C.c_void_p(_ptr(u)),
                                                         str(path).encode()))

    def L2Error(self, u, kind: int, params, t: float = 0.0) -> np.ndarray:
        """MeshFn::L2Error (src/MeshFn.cpp:283-296) against the analytic field
        (kind, params) at time t, per component."""
        p = np.zeros(8)
        p[: len(params)] = params
        out = np.zeros(4)
        self.ctx.check(self._lib.cpg_l2error(self.ctx.h, self.h, C.c_void_p(_ptr(u)), kind, _pd(p), t, _pd(out)))
        return out[: self.nc]

    def __del__(self):
        try:
            if self.h:
                self._lib.cpg_equation_destroy(self.h)
                self.h = None
        except Exception:
            pass


def Advection(ctx, msh, degree, **kw):
    """Advection with beta = (2y-1, -2x+1) (eqns/Advection.cpp:8-16)."""
    return Equation(ctx, msh, ADVECTION_ROTATING, degree, **kw)


def ConstantAdvection(ctx, msh, degree, bx, by, **kw):
    return Equation(ctx, msh, ADVECTION_CONST, degree, beta=(bx, by), **kw)


def Euler(ctx, msh, degree, gamma=1.4, **kw):
    return Equation(ctx, msh, EULER, degree, gamma=gamma, **kw)


class BlockMatrix:
    """Block sparse matrix (BlockMatrix, src/BlockMatrix.h)."""

    def __init__(self, ctx: Context, handle):
        self.ctx = ctx
        self._lib = ctx._lib
        self.h = handle
        n, bl, nnzb, prec = C.c_int(), C.c_int(), C.c_int64(), C.c_int()
        self._lib.cpg_bsr_get_info(self.h, C.byref(n), C.byref(bl), C.byref(nnzb), C.byref(prec))
        self.n_rows, self.bl, self.nb, self.precision = n.value, bl.value, nnzb.value, prec.value

    @classmethod
    def from_host(cls, ctx: Context, rowptr, colidx, blocks=None, bl=None, precision: int = F64):
        rowptr = np.ascontiguousarray(rowptr, np.int32)
        colidx = np.ascontiguousarray(colidx, np.int32)
        if blocks is not None:
            blocks = np.ascontiguousarray(blocks, np.float64)
            bl = blocks.shape[-1]
        h = C.c_void_p()
        ctx.check(ctx._lib.cpg_bsr_create_host(ctx.h, len(rowptr) - 1, bl, _pi(rowptr), _pi(colidx),
                                               None if blocks is None else _pd(blocks), precision, C.byref(h)))
        return cls(ctx, h)

    def export(self):
        """(rowptr, colidx, blocks[nnzb, bl, bl]) with blocks[k][c][r] = A_k(r, c)."""
        rp = np.zeros(self.n_rows + 1, np.int32)
        cl = np.zeros(self.nb, np.int32)
        vals = np.zeros((self.nb, self.bl, self.bl))
        self.ctx.check(self._lib.cpg_bsr_export(self.ctx.h, self.h, _pi(rp), _pi(cl), _pd(vals)))
        return rp, cl, vals

    def spy(self, path: str) -> None:
        """BlockMatrix::spy: nonzero entries as gnuplot text."""
        self.ctx.check(self._lib.cpg_bsr_write_spy(self.ctx.h, self.h, str(path).encode()))

    def matvec(self, x):
        import torch
        y = torch.empty_like(x)
        self.ctx.check(self._lib.cpg_bsr_matvec(self.ctx.h, self.h, C.c_void_p(_ptr(x)), C.c_void_p(_ptr(y))))
        return y

    def gmres(self, b, x, m: int, tol: float, maxIt: int, pc: "Preconditioner | None" = None,
              flexible: bool = False):
        """Solve A x = b; x holds the initial guess.  Returns (its, tol)."""
        st = _capi.SolveStats()
        self.ctx.check(self._lib.cpg_gmres(self.ctx.h, self.h, pc.h if pc is not None else None,
                                           C.c_void_p(_ptr(b)), C.c_void_p(_ptr(x)), m, tol, maxIt, int(flexible),
                                           C.byref(st)))
        return st.iterations, st.residual

    @classmethod
    def stack(cls, parts) -> "BlockMatrix":
        """Block-diagonal stack of matrices of one block size and precision;
        .seg_rows holds each part's first block row (and the total)."""
        parts = list(parts)
        ctx = parts[0].ctx
        arr = (C.c_void_p * len(parts))(*[p.h.value if isinstance(p.h, C.c_void_p) else p.h for p in parts])
        h = C.c_void_p()
        ctx.check(ctx._lib.cpg_bsr_stack(ctx.h, len(parts), arr, C.byref(h)))
        out = cls(ctx, h)
        out.seg_rows = np.cumsum([0] + [p.n_rows for p in parts]).astype(np.int32)
        return out

    def gmres_batched(self, seg_rows, b, x, m: int, tol: float, maxIt: int, pc: "Preconditioner | None" = None,
                      flexible: bool = False):
        """Independent systems on the diagonal blocks [seg_rows[k],
        seg_rows[k+1]) solved together; returns [(its, tol)] per system."""
        seg = np.ascontiguousarray(seg_rows, dtype=np.int32)
        K = len(seg) - 1
        st = (_capi.SolveStats * K)()
        self.ctx.check(self._lib.cpg_gmres_batched(self.ctx.h, self.h, pc.h if pc is not None else None, K, _pi(seg),
                                                   C.c_void_p(_ptr(b)), C.c_void_p(_ptr(x)), m, tol, maxIt,
                                                   int(flexible), st))
        return [(s.iterations, s.residual) for s in st]

    def jacobi(self, b, x, tol: float, maxIt: int, pc: "BlockJacobi"):
        st = _capi.SolveStats()
        self.ctx.check(self._lib.cpg_jacobi_solve(self.ctx.h, self.h, pc.h, C.c_void_p(_ptr(b)),
                                                  C.c_void_p(_ptr(x)), tol, maxIt, C.byref(st)))
        return st.iterations, st.residual

    def __del__(self):
        try:
            if self.h:
                self._lib.cpg_bsr_destroy(self.h)
                self.h = None
        except Exception:
            pass


class Jacobian(BlockMatrix):
    """Jacobian (src/Jacobian.h): a BlockMatrix with the mesh pattern."""

    @classmethod
    def for_equation(cls, eq: Equation, precision: int = F64):
        h = C.c_void_p()
        eq.ctx.check(eq._lib.cpg_bsr_create(eq.ctx.h, eq.h, precision, C.byref(h)))
        return cls(eq.ctx, h)


class Preconditioner:
    kind = PC_NONE

    def __init__(self, A: BlockMatrix, precision: int = F64):
        self.ctx = A.ctx
        self._lib = A._lib
        h = C.c_void_p()
        self.ctx.check(self._lib.cpg_precond_create(self.ctx.h, A.h, self.kind, precision, C.byref(h)))
        self.h = h
        self.n, self.bl, self.precision = A.n_rows, A.bl, precision

    def refactor(self, A: BlockMatrix):
        self.ctx.check(self._lib.cpg_precond_refactor(self.ctx.h, self.h, A.h))

    def solve(self, x):
        """Preconditioner::solve: x <- P^{-1} x in place."""
        self.ctx.check(self._lib.cpg_precond_apply(self.ctx.h, self.h, C.c_void_p(_ptr(x))))
        return x

    def apply_op(self, A: BlockMatrix, x, accuracy: float = 0.0):
        """P^{-1} A x, the operator of a left-preconditioned GMRES step; the
        split form when this is an FP64 ILU(0) of A's current values and
        0.25 eps pivot_cond() <= accuracy (0: the plain product)."""
        import torch
        y = torch.empty_like(x)
        self.ctx.check(self._lib.cpg_precond_apply_op(self.ctx.h, self.h, A.h, C.c_void_p(_ptr(x)),
                                                      C.c_void_p(_ptr(y)), accuracy))
        return y

    def split_ready(self, A: BlockMatrix) -> bool:
        return bool(self._lib.cpg_precond_split_ready(self.h, A.h))

    def pivot_cond(self) -> float:
        """largest cond_inf of a pivot block in the last factorisation"""
        return float(self._lib.cpg_precond_pivot_cond(self.h))

    def levels(self):
        nl, nu = C.c_int(), C.c_int()
        self._lib.cpg_precond_levels(self.h, C.byref(nl), None, None, C.byref(nu), None, None)
        lp, lr = np.zeros(nl.value + 1, np.int32), np.zeros(self.n, np.int32)
        up, ur = np.zeros(nu.value + 1, np.int32), np.zeros(self.n, np.int32)
        self._lib.cpg_precond_levels(self.h, C.byref(nl), _pi(lp), _pi(lr), C.byref(nu), _pi(up), _pi(ur))
        return lp, lr, up, ur

    def export(self, nnz_l: int, nnz_u: int):
        b = self.bl
        dd = np.zeros((self.n, b, b))
        lrp, urp = np.zeros(self.n + 1, np.int32), np.zeros(self.n + 1, np.int32)
        lc, uc = np.zeros(max(nnz_l, 1), np.int32), np.zeros(max(nnz_u, 1), np.int32)
        lv, uv = np.zeros((max(nnz_l, 1), b, b)), np.zeros((max(nnz_u, 1), b, b))
        self.ctx.check(self._lib.cpg_precond_export(self.ctx.h, self.h, _pd(dd), _pi(lrp), _pi(lc), _pd(lv),
                                                    _pi(urp), _pi(uc), _pd(uv)))
        return dd, (lrp, lc[:nnz_l], lv[:nnz_l]), (urp, uc[:nnz_u], uv[:nnz_u])

    def __del__(self):
        try:
            if self.h:
                self._lib.cpg_precond_destroy(self.h)
                self.h = None
        except Exception:
            pass


class NoPreconditioner(Preconditioner):
    kind = PC_NONE


class BlockJacobi(Preconditioner):
    kind = PC_BJACOBI


class BlockILU0(Preconditioner):
    kind = PC_ILU0


class TimeStepper:
    """TimeStepper::advance (src/TimeIntegration.h:16) on device fields."""
    kind = STEP_RK4

    def __init__(self, eq: Equation, kind: int | None = None, pc: int = PC_ILU0, precision: int = F64,
                 gmres_m: int = 20, gmres_tol: float = 1e-14, gmres_maxit: int = 0, flexible: bool = False,
                 newton_tol: float = 5e-13, newton_maxit: int = 100, reuse_jacobian: int = 0,
                 newton_rtol: float = 0.0, pc_f32: bool = False):
        self.eq = eq
        self.ctx = eq.ctx
        self._lib = eq._lib
        d = _capi.StepperDesc()
        d.kind = self.kind if kind is None else kind
        d.pc_kind = pc
        d.matrix_precision = precision
        d.gmres_m = gmres_m
        d.gmres_tol = gmres_tol
        d.gmres_maxit = gmres_maxit
        d.flexible = int(flexible)
        d.newton_tol = newton_tol
        d.newton_maxit = newton_maxit
        d.reuse_jacobian = reuse_jacobian
        d.newton_rtol = newton_rtol
        d.pc_f32 = int(pc_f32)
        h = C.c_void_p()
        self.ctx.check(self._lib.cpg_stepper_create(self.ctx.h, eq.h, C.byref(d), C.byref(h)))
        self.h = h
        self.stats = _capi.StepStats()

    def advance(self, u, dt: float, t: float = 0.0):
        """u <- advance(u, dt, t) in place on the device; returns u."""
        self.ctx.check(self._lib.cpg_step(self.ctx.h, self.h, C.c_void_p(_ptr(u)), dt, t, C.byref(self.stats)))
        return u

    def advance_host(self, u_host: np.ndarray, dt: float, t: float = 0.0) -> np.ndarray:
        """same with a host (numpy float64) field, copied in and out."""
        assert u_host.dtype == np.float64 and u_host.flags.c_contiguous
        self.ctx.check(self._lib.cpg_step_host(self.ctx.h, self.h, _pd(u_host), dt, t, C.byref(self.stats)))
        return u_host

    def __del__(self):
        try:
            if self.h:
                self._lib.cpg_stepper_destroy(self.h)
                self.h = None
        except Exception:
            pass


class ForwardEuler(TimeStepper):
    kind = STEP_FORWARD_EULER


class RK2(TimeStepper):
    kind = STEP_RK2


class RK4(TimeStepper):
    kind = STEP_RK4


class BackwardEuler(TimeStepper):
    kind = STEP_BACKWARD_EULER


class DIRK(TimeStepper):
    """DIRK::advance (src/TimeIntegration.cpp:93-151).  nStages = 3 is the
    reference's tableau (getDIRK, :70-77: order 2, not A-stable); pass
    l_stable=True for Alexander's L-stable SDIRK3 (same as SDIRK3)."""

    def __init__(self, nStages: int, eq: Equation, l_stable: bool = False, **kw):
        if l_stable and nStages != 3:
            raise ValueError("the L-stable tableau has 3 stages")
        self.kind = STEP_SDIRK3 if l_stable else {3: STEP_DIRK3, 5: STEP_DIRK5}[nStages]
        super().__init__(eq, **kw)


class SDIRK3(TimeStepper):
    """Alexander's L-stable 3-stage SDIRK of order 3 on the DIRK::advance
    Newton/GMRES path (the reference's DIRK3 with an A-stable tableau)."""
    kind = STEP_SDIRK3


class IRK(TimeStepper):
    def __init__(self, nStages: int, eq: Equation, inverted: bool = False, **kw):
        self.kind = {(2, False): STEP_IRK2, (3, False): STEP_IRK3, (2, True): STEP_IRK2_INV,
                     (3, True): STEP_IRK3_INV}[(nStages, inverted)]
        super().__init__(eq, **kw)
