"""Known-answer tests that pin the oracle (the reference ships no test,
fixture or golden vector, and cannot be built here).  Each test fixes a
piece of the restated reference arithmetic to mathematics independent of
this project's code: numpy's Legendre module and dense LAPACK solves,
closed-form integrals, conservation and linearity identities, and
temporal convergence orders."""
import numpy as np
import numpy.polynomial.legendre as npleg
import pytest

import cpolyg_b200 as cp
import oracle
from cases import mesh


def idx_pairs(p):
    return [(i, j) for i in range(p + 1) for j in range(p + 1 - i)]


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5])
def test_leg2d_matches_numpy(p):
    rng = np.random.default_rng(p)
    pairs = idx_pairs(p)
    c = rng.standard_normal(len(pairs))
    for x, y in rng.uniform(-1, 1, (20, 2)):
        ref = sum(ck * npleg.legval(x, np.eye(p + 1)[i]) * npleg.legval(y, np.eye(p + 1)[j])
                  for ck, (i, j) in zip(c, pairs))
        assert abs(oracle.leg2d(x, y, p + 1, c) - ref) < 1e-13 * max(1, abs(ref))


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5])
def test_legder_matches_analytic(p):
    """LegDerX/LegDerY (Legendre.cpp:34-124) give the exact derivative series."""
    rng = np.random.default_rng(10 + p)
    pairs = idx_pairs(p)
    c = rng.standard_normal(len(pairs))
    dx, dy = oracle.legder(p + 1, c)
    for x, y in rng.uniform(-1, 1, (10, 2)):
        ex = sum(ck * npleg.legval(x, npleg.legder(np.eye(p + 1)[i])) * npleg.legval(y, np.eye(p + 1)[j])
                 for ck, (i, j) in zip(c, pairs))
        ey = sum(ck * npleg.legval(x, np.eye(p + 1)[i]) * npleg.legval(y, npleg.legder(np.eye(p + 1)[j]))
                 for ck, (i, j) in zip(c, pairs))
        assert abs(oracle.leg2d(x, y, p + 1, dx) - ex) < 1e-12 * max(1, abs(ex))
        assert abs(oracle.leg2d(x, y, p + 1, dy) - ey) < 1e-12 * max(1, abs(ey))


def exact_tri_monomial(T, a, b):
    # integral of x^a y^b over a triangle via a high-order tensor Gauss rule
    # on the collapsed square (exact for polynomials)
    x1, y1, x2, y2, x3, y3 = T
    g, w = npleg.leggauss(20)
    s = 0.5 * (g + 1)
    tot = 0.0
    for si, wi in zip(s, w):
        for ti, wj in zip(s, w):
            u, v = si * (1 - ti), si * ti
            x = x1 + (x2 - x1) * u + (x3 - x1) * v
            y = y1 + (y2 - y1) * u + (y3 - y1) * v
            jac = abs((x2 - x1) * (y3 - y1) - (x3 - x1) * (y2 - y1)) * si
            tot += 0.25 * wi * wj * jac * x ** a * y ** b
    return tot


@pytest.mark.parametrize("deg", [2, 4, 6, 8])
def test_triangle_rules_exact(deg):
    """Quadrature.cpp tables: exact for total degree <= rule degree (to the
    tables' 14 digits)."""
    T = [0.1, 0.2, 0.9, 0.35, 0.3, 0.8]
    for a in range(deg + 1):
        for b in range(deg + 1 - a):
            ex = exact_tri_monomial(T, a, b)
            assert abs(oracle.tri_integral(T, deg, a, b) - ex) < 5e-13


@pytest.mark.parametrize("deg,npts", [(2, 2), (4, 4), (6, 6), (8, 10)])
def test_line_rules_exact(deg, npts):
    x1, y1, x2, y2 = 0.2, 0.1, 0.7, 0.9
    L = np.hypot(x2 - x1, y2 - y1)
    g, w = npleg.leggauss(30)
    for a in range(2 * npts):
        for b in range(2 * npts - a):
            t = 0.5 * (g + 1)
            x, y = x1 + t * (x2 - x1), y1 + t * (y2 - y1)
            ex = 0.5 * L * np.sum(w * x ** a * y ** b)
            assert abs(oracle.line_integral(x1, y1, x2, y2, deg, a, b) - ex) < 1e-13


@pytest.mark.parametrize("m", [1, 2, 3, 4, 5, 8])
def test_gauss_nodes(m):
    assert np.allclose(oracle.gl_nodes(m), npleg.leggauss(m)[0], atol=1e-15, rtol=0)


def rect_mesh(nx, ny, W=1.0, H=1.0, periodic=False):
    polys = []
    for j in range(ny):
        for i in range(nx):
            x0, y0, hx, hy = i * W / nx, j * H / ny, W / nx, H / ny
            polys.append([(x0, y0), (x0 + hx, y0), (x0 + hx, y0 + hy), (x0, y0 + hy)])
    return cp.PolyMesh.from_polygons(polys, W, H, periodic=periodic)


@pytest.mark.parametrize("p", [1, 2, 3])
def test_mass_matrix_rectangle_closed_form(p):
    """Axis-aligned rectangle: M = |K| diag(1 / ((2i+1)(2j+1)))."""
    m = rect_mesh(3, 2, 1.5, 1.0)
    om = oracle.Mesh(m.export())
    eq = oracle.Equation(om, 0, p)
    M = eq.mass_blocks()
    area = 0.5 * (1.0 / 2)
    ref = np.diag([area / ((2 * i + 1) * (2 * j + 1)) for i, j in idx_pairs(p)])
    for i in range(om.n):
        assert np.abs(M[i] - ref).max() < 2e-13


@pytest.mark.parametrize("deg", [1, 2, 3])
def test_free_stream_preserved(deg):
    """Constant Euler state on a periodic Voronoi mesh: zero residual."""
    _, a, om = mesh(400, True, 1.0)
    eq = oracle.Equation(om, 2, deg)
    U = eq.interp(0, [1.2, 0.3, -0.4, 3.1])
    assert np.abs(eq.assemble(U)).max() < 1e-12


@pytest.mark.parametrize("phys", [0, 1])
def test_advection_linearity(phys):
    """Advection is linear: J u = assemble(u) (Equation::jacobian is exact)."""
    _, a, om = mesh(400, phys == 0, 1.0)
    eq = oracle.Equation(om, phys, 2, beta=(0.7, -1.1), dkind=0, dparams=[0.0])
    u = np.random.default_rng(0).standard_normal(eq.ndof)
    rp, cl, blk = eq.jacobian(u)
    assert np.abs(oracle.bsr_matvec(rp, cl, blk, u) - eq.assemble(u)).max() < 1e-12 * np.abs(u).max()


def test_euler_diagonal_blocks_match_finite_differences():
    """Diagonal Jacobian blocks are the exact derivative of the residual
    (off-diagonal blocks use A(u_own), the reference's approximation)."""
    _, a, om = mesh(120, True, 10.0)
    eq = oracle.Equation(om, 2, 2)
    rng = np.random.default_rng(1)
    U = eq.interp(2, [5.0, 5.0, 5.0, 1.0, 1.0, 1.4, 10.0, 10.0])
    U = U * (1 + 0.05 * rng.standard_normal(U.size))  # cell-wise jumps
    rp, cl, blk = eq.jacobian(U)
    bl = eq.bl
    for dof in [0, 5, 13, 17, 26, 40]:
        cell, c = dof // bl, dof % bl
        h = 1e-6 * max(1.0, abs(U[dof]))
        e = np.zeros(U.size)
        e[dof] = h
        fd = (eq.assemble(U + e) - eq.assemble(U - e)) / (2 * h)
        col = blk[rp[cell]][c]
        assert np.abs(fd[cell * bl:(cell + 1) * bl] - col).max() < 1e-5 * np.abs(col).max()


def test_euler_jacobian_defect_and_exact_mode():
    """The reference's A_x entry (3,1) is H - (g-1)(u^2+v^2) (Euler.cpp:154-163)
    where d((rhoE+p)u)/d(rho u) = H - (g-1)u^2; on a smooth state its
    Jacobian is therefore a few percent off.  The exact mode (that entry
    fixed, neighbour blocks differentiated with respect to the neighbour
    state) matches finite differences in every block."""
    _, a, om = mesh(150, True, 10.0)
    V = [5.0, 5.0, 5.0, 1.0, 1.0, 1.4, 10.0, 10.0]
    errs = {}
    for exact in (False, True):
        eq = oracle.Equation(om, 2, 2, dkind=2, dparams=V, exact_jacobian=exact)
        U = eq.interp(2, V)
        rp, cl, blk = eq.jacobian(U)
        n, bl = eq.n, eq.bl
        worst = 0.0
        for dof in np.random.default_rng(0).choice(n * bl, 10, replace=False):
            h = 1e-7
            e = np.zeros(n * bl)
            e[dof] = h
            fd = (eq.assemble(U + e) - eq.assemble(U - e)) / (2 * h)
            col = np.zeros(n * bl)
            cell, c = dof // bl, dof % bl
            for i in range(n):
                for k in range(rp[i], rp[i + 1]):
                    if cl[k] == cell:
                        col[i * bl:(i + 1) * bl] = blk[k][c]
            worst = max(worst, np.abs(fd - col).max() / np.abs(col).max())
        errs[exact] = worst
    assert errs[True] < 1e-6
    assert errs[False] > 1e-3


def test_exact_jacobian_converges_to_the_same_solution():
    """Newton with exact or reference Jacobians converges to the same stage
    values (the residual is unchanged); the exact one in fewer iterations."""
    _, a, om = mesh(300, True, 10.0, 2)
    V = [5.0, 5.0, 5.0, 1.0, 1.0, 1.4, 10.0, 10.0]
    out = {}
    for exact in (False, True):
        eq = oracle.Equation(om, 2, 2, dkind=2, dparams=V, exact_jacobian=exact)
        st = oracle.Stepper(eq, 4, pc=2, gmres_m=30, gmres_tol=1e-10)
        out[exact] = (st.advance(eq.interp(2, V), 0.05), int(st.stats[0]))
    assert np.linalg.norm(out[True][0] - out[False][0]) / np.linalg.norm(out[False][0]) < 1e-11
    assert out[True][1] < out[False][1]


def test_ilu0_is_exact_lu_on_block_tridiagonal():
    """On a 1D chain (no fill outside the pattern) ILU(0) = exact LU."""
    rng = np.random.default_rng(2)
    n, bl = 12, 5
    rp, cl, blocks = [0], [], []
    for i in range(n):
        for j in (i, i - 1, i + 1):  # diagonal first, as the Jacobian pattern
            if 0 <= j < n:
                cl.append(j)
                B = rng.standard_normal((bl, bl))
                blocks.append(B + (4 * bl * np.eye(bl) if i == j else 0))
        rp.append(len(cl))
    blocks = np.array(blocks)
    A = np.zeros((n * bl, n * bl))
    for i in range(n):
        for k in range(rp[i], rp[i + 1]):
            A[i * bl:(i + 1) * bl, cl[k] * bl:(cl[k] + 1) * bl] = blocks[k].T
    x = rng.standard_normal(n * bl)
    z = oracle.precond_apply(2, rp, cl, blocks, x)
    assert np.abs(z - np.linalg.solve(A, x)).max() < 1e-12 * np.abs(np.linalg.solve(A, x)).max()
    z = oracle.precond_apply(1, rp, cl, blocks, x)  # block Jacobi = block-diagonal solve
    for i in range(n):
        D = blocks[rp[i]].T
        assert np.allclose(z[i * bl:(i + 1) * bl], np.linalg.solve(D, x[i * bl:(i + 1) * bl]), rtol=1e-12,
                           atol=1e-14)


def test_gmres_matches_dense_solve():
    rng = np.random.default_rng(3)
    _, a, om = mesh(80, True, 1.0, 2)
    eq = oracle.Equation(om, 0, 1)
    rp, cl, _ = eq.jacobian(np.zeros(eq.ndof))
    bl = 4
    blocks = rng.standard_normal((len(cl), bl, bl))
    for i in range(len(rp) - 1):
        blocks[rp[i]] += 3 * bl * np.eye(bl)
    n = len(rp) - 1
    A = np.zeros((n * bl, n * bl))
    for i in range(n):
        for k in range(rp[i], rp[i + 1]):
            A[i * bl:(i + 1) * bl, cl[k] * bl:(cl[k] + 1) * bl] += blocks[k].T
    b = rng.standard_normal(n * bl)
    for pc in (0, 1, 2):
        x, its, res = oracle.gmres(pc, rp, cl, blocks, b, np.zeros_like(b), 20, 1e-13, 5000)
        assert np.abs(x - np.linalg.solve(A, b)).max() < 1e-10
        assert res < 1e-13 and its > 0


@pytest.mark.parametrize("p", [1, 2, 3])
def test_interp_reproduces_polynomials(p):
    _, a, om = mesh(50, False, 1.0, 4)
    eq = oracle.Equation(om, 0, p)
    # projection of a constant is exact and cell-local: c0 = value, rest 0
    u = eq.interp(0, [2.5]).reshape(om.n, -1)
    assert np.abs(u[:, 0] - 2.5).max() < 1e-13 and np.abs(u[:, 1:]).max() < 1e-13
    # L2 norm of 1 = sqrt(area)
    one = eq.interp(0, [1.0])
    assert abs(eq.l2norm(one)[0] - 1.0) < 1e-12


def temporal_error(kind, dts, T, p=2, n=200):
    _, a, om = mesh(n, True, 1.0, 6)
    eq = oracle.Equation(om, 0, p, beta=(1.0, 0.5))
    u0 = eq.interp(1, [10.0, 0.5, 0.5])
    outs = []
    for dt in dts:
        st = oracle.Stepper(eq, kind, pc=2, gmres_m=30, gmres_tol=1e-14, gmres_maxit=2000, newton_tol=1e-13)
        u, t = u0.copy(), 0.0
        for _ in range(int(round(T / dt))):
            u = st.advance(u, dt, t)
            t += dt
        outs.append(u)
    return outs


def test_rk4_fourth_order():
    u = temporal_error(2, [0.004, 0.002, 0.001], 0.04)
    r = np.linalg.norm(u[0] - u[1]) / np.linalg.norm(u[1] - u[2])
    assert 12 < r < 22


def test_dirk3_tableau_is_second_order():
    """The reference's 3-stage DIRK (TimeIntegration.cpp:70-77) is Crouzeix's
    tableau evaluated with alpha = 0.435866521508459 instead of
    2 cos(pi/18)/sqrt(3); it meets the order-2 conditions but not
    sum b A c = 1/6.  The oracle and the GPU keep the reference's constants,
    so the observed temporal order is 2."""
    a = 0.435866521508459
    A = np.array([[(1 + a) / 2, 0, 0], [-a / 2, (1 + a) / 2, 0], [1 + a, -(1 + 2 * a), (1 + a) / 2]])
    b = np.array([1 / 6 / a ** 2, 1 - 1 / 3 / a ** 2, 1 / 6 / a ** 2])
    c = A.sum(1)
    assert abs(b.sum() - 1) < 1e-15 and abs(b @ c - 0.5) < 1e-15
    assert abs(b @ A @ c - 1 / 6) > 0.3
    u = temporal_error(4, [0.004, 0.002, 0.001], 0.016)
    r = np.linalg.norm(u[0] - u[1]) / np.linalg.norm(u[1] - u[2])
    assert 3 < r < 5


def _tableau(kind):
    """(A, b) of the implicit tableaux, written out independently of the
    oracle and the library (src/TimeIntegration.cpp:68-186)."""
    r6 = np.sqrt(6.0)
    if kind == "dirk3_reference":
        a = 0.435866521508459
        A = [[(1 + a) / 2, 0, 0], [-a / 2, (1 + a) / 2, 0], [1 + a, -(1 + 2 * a), (1 + a) / 2]]
        b = [1 / 6 / a ** 2, 1 - 1 / 3 / a ** 2, 1 / 6 / a ** 2]
    elif kind == "sdirk3":
        g = 0.435866521508459
        b1, b2 = -(6 * g * g - 16 * g + 1) / 4, (6 * g * g - 20 * g + 5) / 4
        A = [[g, 0, 0], [(1 - g) / 2, g, 0], [b1, b2, g]]
        b = [b1, b2, g]
    elif kind == "backward_euler":
        A, b = [[1.0]], [1.0]
    elif kind == "dirk5":
        g = (6 - r6) / 10
        A = [[g, 0, 0, 0, 0], [(-6 + 5 * r6) / 14, g, 0, 0, 0],
             [(888 + 607 * r6) / 2850, (126 - 161 * r6) / 1425, g, 0, 0],
             [(3153 - 3082 * r6) / 14250, (3213 + 1148 * r6) / 28500, (-267 + 88 * r6) / 500, g, 0],
             [(-32583 + 14638 * r6) / 71250, (-17199 + 364 * r6) / 142500, (1329 - 544 * r6) / 2500,
              (-96 + 131 * r6) / 625, g]]
        b = [0, 0, 1 / 9, (16 - r6) / 36, (16 + r6) / 36]
    elif kind == "radau2":
        A, b = [[5 / 12, -1 / 12], [3 / 4, 1 / 4]], [3 / 4, 1 / 4]
    else:  # radau3
        A = [[(88 - 7 * r6) / 360, (296 - 169 * r6) / 1800, (-2 + 3 * r6) / 225],
             [(296 + 169 * r6) / 1800, (88 + 7 * r6) / 360, (-2 - 3 * r6) / 225],
             [(16 - r6) / 36, (16 + r6) / 36, 1 / 9]]
        b = [(16 - r6) / 36, (16 + r6) / 36, 1 / 9]
    return np.array(A, dtype=np.float64), np.array(b, dtype=np.float64)


def stability(A, b, z):
    """R(z) = 1 + z b^T (I - zA)^{-1} 1"""
    s = len(b)
    return 1 + z * b @ np.linalg.solve(np.eye(s) - z * A, np.ones(s))


@pytest.mark.parametrize("kind", ["sdirk3", "backward_euler", "dirk5", "radau2", "radau3"])
def test_implicit_tableaux_are_a_stable(kind):
    """|R(z)| <= 1 on the closed left half-plane for every implicit tableau a
    benchmark runs.  R is rational with poles at the reciprocals of A's
    eigenvalues; with all of them in the right half-plane, the maximum
    principle reduces the check to the imaginary axis (sampled densely, plus
    z -> infinity along the negative real axis)."""
    A, b = _tableau(kind)
    assert (np.linalg.eigvals(A).real > 0).all()
    ys = np.concatenate([np.linspace(-50, 50, 20001), np.geomspace(50, 1e8, 2000)])
    mx = max(abs(stability(A, b, 1j * y)) for y in np.concatenate([ys, -ys]))
    assert mx <= 1 + 1e-12
    assert abs(stability(A, b, -1e12)) <= 1.0


def test_reference_dirk3_tableau_is_not_a_stable():
    """The reference's getDIRK(3) amplifies stiff modes: |R(-inf)| = 1.78 and
    |R(-10)| = 1.20, so at the 100k-cell vortex's time step (CFL ~ 50 for the
    p=3 modes) the scheme is unstable; benchmarks run SDIRK3 instead."""
    A, b = _tableau("dirk3_reference")
    assert abs(stability(A, b, -1e12)) > 1.7
    assert abs(stability(A, b, -10.0)) > 1.15


def test_sdirk3_is_third_order_and_l_stable():
    """Alexander's SDIRK3: order-3 conditions, stiffly accurate, R(-inf) = 0;
    the oracle's temporal order on advection is 3 (error ratio ~8 per
    halving of dt)."""
    A, b = _tableau("sdirk3")
    c = A.sum(1)
    assert abs(b.sum() - 1) < 1e-14 and abs(b @ c - 1 / 2) < 1e-14
    assert abs(b @ c ** 2 - 1 / 3) < 1e-14 and abs(b @ A @ c - 1 / 6) < 1e-14
    assert np.array_equal(A[-1], b)
    assert abs(stability(A, b, -1e12)) < 1e-6
    u = temporal_error(10, [0.004, 0.002, 0.001], 0.016)
    r = np.linalg.norm(u[0] - u[1]) / np.linalg.norm(u[1] - u[2])
    assert 6.5 < r < 9.5


def test_radau_iia_third_order():
    u = temporal_error(6, [0.004, 0.002, 0.001], 0.016)
    r = np.linalg.norm(u[0] - u[1]) / np.linalg.norm(u[1] - u[2])
    assert 6 < r < 10


def test_l2error_of_zero_field_is_the_exact_norm():
    """MeshFn::L2Error of the zero field is the L2 norm of the exact field:
    for exp(-a r^2) well inside the periodic unit square that is
    sqrt(pi / (2a)); the moving, wrapped centre gives the same value."""
    _, a, om = mesh(1000, True, 1.0, 1)
    eq = oracle.Equation(om, 0, 3, beta=(1.0, 1.0))
    z = np.zeros(eq.ndof)
    a_ = 100.0
    want = np.sqrt(np.pi / (2 * a_))
    e0 = eq.l2error(z, 1, [a_, 0.5, 0.5])[0]
    e1 = eq.l2error(z, 1, [a_, 0.1, 0.2, 1.0, 1.0, 1.0, 1.0], t=0.4)[0]  # centre (0.5, 0.6)
    assert abs(e0 - want) < 1e-3 * want and abs(e1 - want) < 1e-3 * want
    # the interpolant of a constant state has no error
    u = eq.interp(0, [0.7])
    assert eq.l2error(u, 0, [0.7])[0] < 1e-13
