"""ctypes binding of include/cpolyg.h (the library's C ABI).

The shared library is the in-tree build ``cpolyg_b200/_lib/libcpolyg_b200.so``.
Loading fails loudly when it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libcpolyg_b200.so")

STATUS = {
    0: "CPG_OK", 1: "CPG_ERR_INVALID_ARG", 2: "CPG_ERR_OOM", 3: "CPG_ERR_SINGULAR_BLOCK",
    4: "CPG_ERR_NONFINITE", 5: "CPG_ERR_NOT_CONVERGED", 6: "CPG_ERR_TIMEOUT", 7: "CPG_ERR_CUDA",
    8: "CPG_ERR_MESH", 9: "CPG_ERR_UNSUPPORTED", 10: "CPG_ERR_NONPHYSICAL",
}

# enums (cpolyg.h)
ADVECTION_CONST, ADVECTION_ROTATING, EULER = 0, 1, 2
BC_DIRICHLET, BC_WALL, BC_OUTFLOW, BC_INFLOW = -1, -2, -3, -4
INIT_CONSTANT, INIT_GAUSSIAN, INIT_VORTEX, INIT_DENSITY_BUMP = 0, 1, 2, 3
F64, F32 = 0, 1
PC_NONE, PC_BJACOBI, PC_ILU0, PC_STAGE_BJACOBI = 0, 1, 2, 3
(STEP_FORWARD_EULER, STEP_RK2, STEP_RK4, STEP_BACKWARD_EULER, STEP_DIRK3, STEP_DIRK5,
 STEP_IRK2, STEP_IRK3, STEP_IRK2_INV, STEP_IRK3_INV, STEP_SDIRK3) = range(11)


class MeshInfo(C.Structure):
    _fields_ = [("n_cells", C.c_int), ("n_verts", C.c_int), ("n_edges", C.c_int), ("n_tris", C.c_int),
                ("periodic", C.c_int), ("width", C.c_double), ("height", C.c_double)]


class EquationDesc(C.Structure):
    _fields_ = [("physics", C.c_int), ("degree", C.c_int), ("gamma", C.c_double), ("beta", C.c_double * 2),
                ("dirichlet_kind", C.c_int), ("dirichlet_params", C.c_double * 8),
                ("inflow_state", C.c_double * 4), ("exact_jacobian", C.c_int)]


class EquationInfo(C.Structure):
    _fields_ = [("n_cells", C.c_int), ("nb", C.c_int), ("nc", C.c_int), ("bl", C.c_int), ("n_dof", C.c_int64),
                ("nnzb", C.c_int64), ("n_vqp", C.c_int), ("n_faces", C.c_int), ("nqf", C.c_int),
                ("levels_lower", C.c_int), ("levels_upper", C.c_int)]


class SolveStats(C.Structure):
    _fields_ = [("iterations", C.c_int), ("residual", C.c_double), ("converged", C.c_int)]


class StepperDesc(C.Structure):
    _fields_ = [("kind", C.c_int), ("pc_kind", C.c_int), ("matrix_precision", C.c_int), ("gmres_m", C.c_int),
                ("gmres_tol", C.c_double), ("gmres_maxit", C.c_int), ("flexible", C.c_int),
                ("newton_tol", C.c_double), ("newton_maxit", C.c_int), ("reuse_jacobian", C.c_int),
                ("newton_rtol", C.c_double), ("pc_f32", C.c_int)]


class StepStats(C.Structure):
    _fields_ = [("newton_iterations", C.c_int), ("gmres_iterations", C.c_int), ("linear_solves", C.c_int),
                ("last_newton_residual", C.c_double), ("converged", C.c_int)]


P = C.c_void_p
I = C.c_int
D = C.c_double
PI = C.POINTER(C.c_int)
PD = C.POINTER(C.c_double)
PP = C.POINTER(C.c_void_p)
I64 = C.c_int64
PI64 = C.POINTER(C.c_int64)

# name -> (restype, argtypes)
PROTOTYPES = {
    "cpg_ctx_create": (I, [I, P, PP]),
    "cpg_ctx_destroy": (None, [P]),
    "cpg_last_error": (C.c_char_p, [P]),
    "cpg_ctx_sync": (I, [P]),
    "cpg_ctx_set_deferred_checks": (I, [P, I]),
    "cpg_ctx_launch_count": (C.c_uint64, [P]),
    "cpg_version": (C.c_char_p, []),
    "cpg_seeds_uniform": (I, [C.c_uint64, I, D, D, PD]),
    "cpg_mesh_voronoi": (I, [PD, I, D, D, I, PI, PP]),
    "cpg_mesh_from_polygons": (I, [I, PI, PD, D, D, I, PI, PP]),
    "cpg_mesh_set_subtriangles": (I, [P, PI, PD]),
    "cpg_mesh_destroy": (None, [P]),
    "cpg_gmres_batched": (I, [P, P, P, I, PI, P, P, I, D, I, I, C.POINTER(SolveStats)]),
    "cpg_bsr_stack": (I, [P, I, PP, PP]),
    "cpg_mesh_write_gnuplot": (I, [P, C.c_char_p]),
    "cpg_field_write_gnuplot": (I, [P, P, P, P, C.c_char_p]),
    "cpg_bsr_write_spy": (I, [P, P, C.c_char_p]),
    "cpg_mesh_get_info": (I, [P, C.POINTER(MeshInfo)]),
    "cpg_mesh_export": (I, [P, PI, PD, PI, PI, PD, PD, PI, PD]),
    "cpg_mesh_pattern": (I, [P, PI, PI, PI64]),
    "cpg_pattern_levels": (I, [I, PI, PI, PI, PI, PI, PI, PI, PI]),
    "cpg_equation_create": (I, [P, P, C.POINTER(EquationDesc), PP]),
    "cpg_equation_destroy": (None, [P]),
    "cpg_equation_get_info": (I, [P, C.POINTER(EquationInfo)]),
    "cpg_assemble": (I, [P, P, P, D, P]),
    "cpg_mass_apply": (I, [P, P, P, P]),
    "cpg_mass_solve": (I, [P, P, P, P]),
    "cpg_l2norm": (I, [P, P, P, PD]),
    "cpg_l2norm_noalloc": (I, [P, P, P, PD]),
    "cpg_l2error": (I, [P, P, P, I, PD, D, PD]),
    "cpg_interp": (I, [P, P, I, PD, D, P]),
    "cpg_mass_export": (I, [P, P, PD]),
    "cpg_bsr_create": (I, [P, P, I, PP]),
    "cpg_bsr_create_host": (I, [P, I, I, PI, PI, PD, I, PP]),
    "cpg_bsr_destroy": (None, [P]),
    "cpg_bsr_get_info": (I, [P, PI, PI, PI64, PI]),
    "cpg_bsr_export": (I, [P, P, PI, PI, PD]),
    "cpg_bsr_upload": (I, [P, P, PD]),
    "cpg_jacobian": (I, [P, P, P, D, D, I, P]),
    "cpg_bsr_matvec": (I, [P, P, P, P]),
    "cpg_precond_create": (I, [P, P, I, I, PP]),
    "cpg_precond_refactor": (I, [P, P, P]),
    "cpg_precond_apply": (I, [P, P, P]),
    "cpg_precond_sweep_form": (I, [P]),
    "cpg_precond_apply_op": (I, [P, P, P, P, P, D]),
    "cpg_precond_split_ready": (I, [P, P]),
    "cpg_precond_pivot_cond": (D, [P]),
    "cpg_debug_sweep_timeout": (I, [P]),
    "cpg_precond_destroy": (None, [P]),
    "cpg_precond_levels": (I, [P, PI, PI, PI, PI, PI, PI]),
    "cpg_precond_export": (I, [P, P, PD, PI, PI, PD, PI, PI, PD]),
    "cpg_gmres": (I, [P, P, P, P, P, I, D, I, I, C.POINTER(SolveStats)]),
    "cpg_jacobi_solve": (I, [P, P, P, P, P, D, I, C.POINTER(SolveStats)]),
    "cpg_axpby": (I, [P, I64, D, P, D, P]),
    "cpg_stepper_create": (I, [P, P, C.POINTER(StepperDesc), PP]),
    "cpg_stepper_destroy": (None, [P]),
    "cpg_step": (I, [P, P, P, D, D, C.POINTER(StepStats)]),
    "cpg_step_host": (I, [P, P, PD, D, D, C.POINTER(StepStats)]),
}

_lib = None


def load() -> C.CDLL:
    """Load the in-tree library (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"cpolyg_b200 CUDA library not built: {LIB_PATH} is missing "
                          "(run `python -m cpolyg_b200.build`)")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in PROTOTYPES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


class CpgError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"{STATUS.get(status, status)}: {msg}")
        self.status = status
