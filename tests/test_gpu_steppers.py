"""Time-stepper parity of the CUDA path against the oracle.

Bar: relative 2-norm difference of the final coefficient vectors
|u_gpu - u_oracle| / |u_oracle| <= 1e-11 for the FP64 path; <= 1e-8 for the
mixed-precision path (FP32 Jacobian and ILU(0) factors, FP64 FGMRES).
"""
import numpy as np
import pytest

import cpolyg_b200 as cp
import oracle
from cases import equations, to_dev, to_np

pytestmark = pytest.mark.gpu


def l2rel(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def run_both(ctx, name, deg, kind, n, width, steps, dt, pc=cp.PC_ILU0, gm=20, gtol=1e-14, gmaxit=90000,
             precision=cp.F64, flexible=False, reuse=0, periodic=True, init=None, codes=None, dirichlet=None,
             inflow=None, oracle_pc=None, exact=False, rtol=0.0):
    # the oracle always runs the reference's Jacobian: an exact-Jacobian GPU
    # run must land on the same converged solution
    ge, oe, _ = equations(ctx, name, deg, n=n, periodic=periodic, width=width, codes=codes, dirichlet=dirichlet,
                          inflow=inflow, exact_jacobian=exact, oracle_exact=False)
    kind_i, params = init
    u0 = oe.interp(kind_i, params)
    ostep = oracle.Stepper(oe, kind, pc=pc if oracle_pc is None else oracle_pc, gmres_m=gm, gmres_tol=gtol,
                           gmres_maxit=gmaxit)
    gstep = cp.TimeStepper(ge, kind=kind, pc=pc, precision=precision, gmres_m=gm, gmres_tol=gtol,
                           gmres_maxit=gmaxit, flexible=flexible, reuse_jacobian=reuse, newton_rtol=rtol)
    uo = u0.copy()
    ug = to_dev(u0).reshape(ge.np, ge.nc, ge.nb)
    t = 0.0
    for _ in range(steps):
        uo = ostep.advance(uo, dt, t)
        gstep.advance(ug, dt, t)
        t += dt
    return to_np(ug), uo, gstep, ostep


GAUSS = (cp.INIT_GAUSSIAN, [100.0, 0.5, 0.5])


@pytest.mark.parametrize("kind", [cp.STEP_FORWARD_EULER, cp.STEP_RK2, cp.STEP_RK4])
def test_explicit_advection(ctx, kind):
    ug, uo, _, _ = run_both(ctx, "adv_const", 2, kind, 1000, 1.0, 20, 1e-4, init=GAUSS)
    assert l2rel(ug, uo) < 1e-11


def test_rk4_config1_full(ctx):
    """Periodic unit square, 1000 Voronoi cells (seed 1), p=2, velocity (1,1),
    u0 = exp(-100 r^2), RK4 dt=1e-4, 200 steps."""
    ug, uo, _, _ = run_both(ctx, "adv_const", 2, cp.STEP_RK4, 1000, 1.0, 200, 1e-4, init=GAUSS)
    assert l2rel(ug, uo) < 1e-11


def test_rk4_euler_vortex(ctx):
    vort = (cp.INIT_VORTEX, [5.0, 5.0, 5.0, 1.0, 1.0, 1.4, 10.0, 10.0])
    ug, uo, _, _ = run_both(ctx, "euler", 2, cp.STEP_RK4, 300, 10.0, 5, 2e-3, init=vort)
    assert l2rel(ug, uo) < 1e-11


VORTEX = (cp.INIT_VORTEX, [5.0, 5.0, 5.0, 1.0, 1.0, 1.4, 10.0, 10.0])


@pytest.mark.parametrize("deg", [2, 3])
def test_dirk3_euler_vortex(ctx, deg):
    """Config-2 semantics at oracle size: periodic [0,10]^2, isentropic vortex
    strength 5, DIRK3 dt=0.05, GMRES(30)+ILU(0) tol 1e-10, Newton 5e-13."""
    ug, uo, gs, os_ = run_both(ctx, "euler", deg, cp.STEP_DIRK3, 150, 10.0, 2, 0.05, gm=30, gtol=1e-10,
                               init=VORTEX)
    assert gs.stats.converged == 1
    assert l2rel(ug, uo) < 1e-11


@pytest.mark.parametrize("deg", [2, 3])
def test_dirk3_exact_jacobian_matches_reference_solution(ctx, deg):
    """The benchmarked configuration: exact Euler Jacobian on the GPU against
    the oracle running the reference's Jacobian; both Newton iterations
    converge to 5e-13, so the stage solutions agree."""
    ug, uo, gs, os_ = run_both(ctx, "euler", deg, cp.STEP_DIRK3, 150, 10.0, 2, 0.05, gm=30, gtol=1e-10,
                               init=VORTEX, exact=True)
    assert gs.stats.converged == 1
    assert l2rel(ug, uo) < 1e-11


def test_backward_euler_and_dirk5_advection(ctx):
    for kind in (cp.STEP_BACKWARD_EULER, cp.STEP_DIRK5):
        ug, uo, _, _ = run_both(ctx, "adv_rot", 2, kind, 200, 1.0, 2, 0.01, gm=20, gtol=1e-12, init=GAUSS,
                                periodic=False, dirichlet=(cp.INIT_CONSTANT, [0.0]))
        assert l2rel(ug, uo) < 1e-11


@pytest.mark.parametrize("kind", [cp.STEP_IRK2, cp.STEP_IRK2_INV, cp.STEP_IRK3])
def test_irk_advection_reference_ilu(ctx, kind):
    """IRK::advance / newAdvance with the reference's BlockILU0 on the
    stage-coupled matrix."""
    ug, uo, gs, _ = run_both(ctx, "adv_const", 2, kind, 150, 1.0, 2, 0.01, gm=20, gtol=1e-12, gmaxit=20000,
                             init=GAUSS)
    assert l2rel(ug, uo) < 1e-11


def test_irk2_euler_stage_block_jacobi(ctx):
    """Config-5 semantics at oracle size: 2-stage Radau IIA, slip walls at
    y=0 and y=H, inflow at x=0, outflow at x=W, density bump in Mach-0.3 flow,
    block Jacobi on the 48x48 cell-coupled stage blocks, GMRES(40) 1e-9."""
    g = 1.4
    inflow = [1.0, 0.3, 0.0, (1.0 / g) / (g - 1) + 0.5 * 0.3 ** 2]
    codes = (cp.BC_WALL, cp.BC_OUTFLOW, cp.BC_WALL, cp.BC_INFLOW)
    bump = (cp.INIT_DENSITY_BUMP, [0.1, 0.5, 5.0, 5.0, 0.3, g])
    ug, uo, gs, _ = run_both(ctx, "euler", 2, cp.STEP_IRK2, 150, 10.0, 1, 0.05, pc=cp.PC_STAGE_BJACOBI, gm=40,
                             gtol=1e-9, gmaxit=20000, init=bump, periodic=False, codes=codes,
                             dirichlet=(cp.INIT_CONSTANT, inflow), inflow=inflow, oracle_pc=3)
    assert gs.stats.converged == 1
    assert l2rel(ug, uo) < 1e-11


def test_mixed_precision_dirk3(ctx):
    """Config-3 semantics: FP32 Jacobian and ILU(0) factors, FP64 FGMRES(30)
    with FP64 residuals; error vs the FP64 oracle <= 1e-8."""
    ug, uo, gs, _ = run_both(ctx, "euler", 3, cp.STEP_DIRK3, 150, 10.0, 2, 0.05, gm=30, gtol=1e-10,
                             precision=cp.F32, flexible=True, init=VORTEX, exact=True)
    assert gs.stats.converged == 1
    assert l2rel(ug, uo) < 1e-8


def test_mixed_precision_dirk3_update_rule(ctx):
    """The FP32-Jacobian Newton iteration converges linearly; requiring the
    last update to be below 1e-10 of the stage vector (newton_rtol) on top of
    the reference's residual rule brings the mixed path to the FP64 oracle's
    converged solution within 1e-10."""
    ug, uo, gs, _ = run_both(ctx, "euler", 3, cp.STEP_DIRK3, 150, 10.0, 2, 0.05, gm=30, gtol=1e-10,
                             precision=cp.F32, flexible=True, init=VORTEX, exact=True, rtol=1e-10)
    assert gs.stats.converged == 1
    assert l2rel(ug, uo) < 1e-10


def test_step_host_matches_device(ctx):
    ge, oe, _ = equations(ctx, "adv_const", 2, n=300)
    u0 = oe.interp(*GAUSS)
    s1 = cp.RK4(ge)
    s2 = cp.RK4(ge)
    ud = to_dev(u0).reshape(ge.np, ge.nc, ge.nb)
    uh = u0.copy()
    for k in range(3):
        s1.advance(ud, 1e-3, k * 1e-3)
        s2.advance_host(uh, 1e-3, k * 1e-3)
    assert np.array_equal(to_np(ud), uh)


def test_explicit_step_graph_replay_matches_direct_launches(ctx):
    """On a context with its own stream, explicit steps are captured once as a
    CUDA graph and replayed; the result must equal the directly launched
    steps of a default-stream context bit for bit, also after dt changes
    (re-capture)."""
    import torch
    ge, oe, _ = equations(ctx, "euler", 2, n=400, periodic=True, width=10.0)
    u0 = to_dev(oe.interp(*VORTEX)).reshape(ge.np, ge.nc, ge.nb)
    direct = cp.RK4(ge)
    ua = u0.clone()
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        sctx = cp.Context(0, stream)
        gs, _, _ = equations(sctx, "euler", 2, n=400, periodic=True, width=10.0)
        graphed = cp.RK4(gs)
        ub = u0.clone()
        launches0, direct0 = sctx.launches, ctx.launches
        t = 0.0
        for dt in (1e-3, 1e-3, 1e-3, 2e-3, 2e-3):
            direct.advance(ua, dt, t)
            graphed.advance(ub, dt, t)
            t += dt
        stream.synchronize()
        # the replays count the kernels they hold
        assert sctx.launches - launches0 == ctx.launches - direct0
    torch.cuda.synchronize()
    assert torch.equal(ua, ub)


# ---------------------------------------------------------------------------
# The benchmark's time step on an oracle-sized mesh: the 100k-cell vortex's
# dt = 0.05 scaled by the cell size (dt = 0.05 * sqrt(100000 / n), the same
# dt/h), 20 steps of Alexander's L-stable SDIRK3, against the oracle's run
# recorded in tests/golden/sdirk3_vortex_p3_1000.npz (make_golden.py).
# ---------------------------------------------------------------------------
def _golden_sdirk3():
    import os

    from golden.make_golden import mesh_digest
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "sdirk3_vortex_p3_1000.npz"))
    m = cp.PolyMesh.voronoi(cp.uniform_seeds(int(g["seed"]), int(g["n"]), 10.0, 10.0), 10.0, 10.0, periodic=True)
    assert mesh_digest(m.export()) == str(g["mesh_sha256"]), "the mesh differs from the one the fixture was made on"
    return g, m


def _run_sdirk3(ctx, g, m, **kw):
    eq = cp.Euler(ctx, m, int(g["degree"]), dirichlet=(cp.INIT_VORTEX, VORTEX[1]), exact_jacobian=True)
    u = eq.interp(cp.INIT_VORTEX, VORTEX[1])
    st = cp.SDIRK3(eq, pc=cp.PC_ILU0, gmres_m=30, gmres_tol=1e-10, gmres_maxit=90000, **kw)
    dt, t, newton = float(g["dt"]), 0.0, []
    for _ in range(int(g["steps"])):
        st.advance(u, dt, t)
        assert st.stats.converged == 1
        newton.append(st.stats.newton_iterations)
        t += dt
    return to_np(u), newton


def test_sdirk3_vortex_20_steps_at_benchmark_cfl(ctx):
    """FP64: <= 1e-11 against the oracle after 20 steps, with the oracle's
    Newton iteration count at every step."""
    g, m = _golden_sdirk3()
    u, newton = _run_sdirk3(ctx, g, m)
    assert l2rel(u, g["u"]) < 1e-11
    assert newton == [int(x) for x in g["newton"]]


def test_sdirk3_vortex_mixed_precision_20_steps(ctx):
    """Mixed precision (FP32 Jacobian and ILU(0) factors, FP64 FGMRES with
    FP64 residuals, Newton update rule 1e-10) stays within 1e-8 of the FP64
    oracle at the final time."""
    g, m = _golden_sdirk3()
    u, _ = _run_sdirk3(ctx, g, m, precision=cp.F32, flexible=True, newton_rtol=1e-10)
    assert l2rel(u, g["u"]) < 1e-8


def test_nonphysical_state_is_reported_by_name(ctx):
    """A negative pressure planted in one cell of the host-built state makes
    the first residual return CPG_ERR_NONPHYSICAL naming that cell (instead of
    a NaN hidden by the flux's max and a singular pivot later), and the
    Rusanov flux carries the NaN sound speed into the residual."""
    import torch
    ge, oe, _ = equations(ctx, "euler", 2, n=200, periodic=True, width=10.0)
    u0 = oe.interp(*VORTEX).reshape(ge.np, ge.nc, ge.nb)
    bad = 37
    u0[bad, 3, 0] = -1.0  # energy below the kinetic energy: p < 0 in the whole cell
    u = to_dev(u0).reshape(ge.np, ge.nc, ge.nb)
    b = torch.empty_like(u)
    with pytest.raises(cp.CpgError) as e:
        ctx.check(ctx._lib.cpg_assemble(ctx.h, ge.h, cp.C.c_void_p(u.data_ptr()), 0.0, cp.C.c_void_p(b.data_ptr())))
    assert e.value.status == 10 and f"cell {bad}" in str(e.value)
    assert not torch.isfinite(b[bad]).all()
    # the context stays usable and the word was cleared: a good state passes
    ug = to_dev(oe.interp(*VORTEX)).reshape(ge.np, ge.nc, ge.nb)
    ge.assemble(ug)
    step = cp.SDIRK3(ge, pc=cp.PC_ILU0, gmres_m=30, gmres_tol=1e-10)
    with pytest.raises(cp.CpgError) as e:
        step.advance(u, 0.05, 0.0)
    assert e.value.status == 10 and f"cell {bad}" in str(e.value) and "Newton iteration 0" in str(e.value)


def test_deferred_checks_report_at_sync(ctx):
    """With deferred checks the residual of a non-physical state returns at
    once and the next cpg_ctx_sync reports it (cell named); afterwards the
    word is clear and checks are immediate again."""
    import torch
    ge, oe, _ = equations(ctx, "euler", 2, n=200, periodic=True, width=10.0)
    u0 = oe.interp(*VORTEX).reshape(ge.np, ge.nc, ge.nb)
    u0[11, 3, 0] = -1.0
    u = to_dev(u0).reshape(ge.np, ge.nc, ge.nb)
    b = torch.empty_like(u)
    lib = ctx._lib
    ctx.check(lib.cpg_ctx_set_deferred_checks(ctx.h, 1))
    try:
        assert lib.cpg_assemble(ctx.h, ge.h, cp.C.c_void_p(u.data_ptr()), 0.0, cp.C.c_void_p(b.data_ptr())) == 0
        with pytest.raises(cp.CpgError) as e:
            ctx.sync()
        assert e.value.status == 10 and "cell 11" in str(e.value)
        ctx.sync()  # cleared
    finally:
        ctx.check(lib.cpg_ctx_set_deferred_checks(ctx.h, 0))
    st = lib.cpg_assemble(ctx.h, ge.h, cp.C.c_void_p(u.data_ptr()), 0.0, cp.C.c_void_p(b.data_ptr()))
    assert st == 10
