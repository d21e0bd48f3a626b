"""Split form of the left-preconditioned Krylov operator P^{-1} A.

For an FP64 block ILU(0) P = (I + L) D (I + U') factored from A (the
reference's BlockILU0: L = L_A D^{-1}, U' = D^{-1} U_A, only the pivot
blocks modified), A = (I + L) D + D U' + E with E_i = A_ii - Ahat_ii, so

    P^{-1} A x = (I + U')^{-1} [x + D^{-1} (I + L)^{-1} (U_A + E) x].

A GMRES step then streams A's upper blocks and E instead of all of A.  The
split product is the plain product of A perturbed by rounding of order
eps * cond(D_i); it is taken only while A holds the values P was factored
from, and by a solve only when 0.25 eps max cond(D_i) is within its
tolerance."""
import pytest
import torch

import cpolyg_b200 as cp

pytestmark = pytest.mark.gpu

V = [5.0, 5.0, 5.0, 1.0, 1.0, 1.4, 10.0, 10.0]
EPS = 2.0 ** -52
GAMMA_SDIRK = 0.435866521508459

# (physics, degree): block sizes 6, 10, 24, 40
CASES = [("advection", 2), ("advection", 3), ("euler", 2), ("euler", 3)]


def rel(a, b) -> float:
    """max |a - b| / max |b| of two device vectors"""
    return ((a - b).abs().max() / b.abs().max()).item()


def newton_system(ctx, physics, degree, n=3000, seed=21):
    """The SDIRK3 stage matrix M - gamma dt J of a vortex (Euler) or a
    Gaussian pulse (constant advection) at the benchmark's CFL number."""
    if physics == "euler":
        m = cp.PolyMesh.voronoi(cp.uniform_seeds(seed, n, 10.0, 10.0), 10.0, 10.0, periodic=True)
        eq = cp.Euler(ctx, m, degree, dirichlet=(cp.INIT_VORTEX, V), exact_jacobian=True)
        u = eq.interp(cp.INIT_VORTEX, V)
        dt = 0.05 * (100000 / n) ** 0.5
    else:
        m = cp.PolyMesh.voronoi(cp.uniform_seeds(seed, n, 1.0, 1.0), 1.0, 1.0, periodic=True)
        eq = cp.ConstantAdvection(ctx, m, degree, 1.0, 1.0)
        u = eq.interp(cp.INIT_GAUSSIAN, [100.0, 0.5, 0.5])
        dt = 0.05
    J = eq.jacobian(u, 0.0, scale=-dt * GAMMA_SDIRK, add_mass=True)
    return eq, u, dt, J


def pair(J, monkeypatch):
    """Two ILU(0) factorisations of J: the plain form and the split form."""
    monkeypatch.setenv("CPG_SPLIT_OPERATOR", "0")
    plain = cp.BlockILU0(J)
    monkeypatch.delenv("CPG_SPLIT_OPERATOR")
    split = cp.BlockILU0(J)
    return plain, split


def rhs(J, seed=5):
    gen = torch.Generator("cuda").manual_seed(seed)
    return torch.randn(J.n_rows * J.bl, dtype=torch.float64, device="cuda", generator=gen)


def prec_residual(J, P, b, x):
    r = b - J.matvec(x)
    return torch.linalg.norm(P.solve(r)).item() / torch.linalg.norm(P.solve(b.clone())).item()


@pytest.mark.parametrize("physics,degree", CASES)
def test_split_operator_matches_plain(ctx, monkeypatch, physics, degree):
    _, _, _, J = newton_system(ctx, physics, degree)
    plain, split = pair(J, monkeypatch)
    assert split.split_ready(J) and not plain.split_ready(J)
    cond = split.pivot_cond()
    assert cond > 1.0 and cond == plain.pivot_cond()
    b = rhs(J)
    y0 = plain.apply_op(J, b, accuracy=1.0)  # not split capable: the plain product
    y1 = split.apply_op(J, b, accuracy=1.0)  # split
    assert not torch.equal(y0, y1)
    assert rel(y1, y0) < 0.25 * EPS * cond, (rel(y1, y0), EPS * cond)
    # accuracy 0: the plain product, bit for bit
    assert torch.equal(split.apply_op(J, b), y0)


@pytest.mark.parametrize("form", [1, 2, 3, 4, 5, 6])
def test_split_backward_add_in_every_sweep_form(ctx, monkeypatch, form):
    """The backward sweep adds x to every row in each of the sweep forms (TMA
    ring, level rows, direct sync-free rows of three widths)."""
    monkeypatch.setenv("CPG_ILU_SWEEP", f"form{form}")
    _, _, _, J = newton_system(ctx, "euler", 3)
    plain, split = pair(J, monkeypatch)
    b = rhs(J)
    y0 = plain.apply_op(J, b)
    y1 = split.apply_op(J, b, accuracy=1.0)
    assert rel(y1, y0) < 0.25 * EPS * split.pivot_cond()


@pytest.mark.parametrize("physics,degree", [("advection", 2), ("euler", 2)])
def test_gmres_takes_the_split_form_where_its_rounding_allows(ctx, monkeypatch, physics, degree):
    _, _, _, J = newton_system(ctx, physics, degree)
    plain, split = pair(J, monkeypatch)
    tol = 1e-10
    assert 0.25 * EPS * split.pivot_cond() <= tol
    b = rhs(J)
    x0, x1 = torch.zeros_like(b), torch.zeros_like(b)
    its0, res0 = J.gmres(b, x0, 30, tol, 9000, plain)
    its1, res1 = J.gmres(b, x1, 30, tol, 9000, split)
    assert not torch.equal(x0, x1)  # the split form ran
    assert res0 < tol and res1 < tol
    assert abs(its1 - its0) <= max(2, its0 // 20), (its0, its1)
    # the split solve's preconditioned residual, measured with plain products
    assert prec_residual(J, plain, b, x1) < 2 * tol
    assert rel(x1, x0) < 1e-8, rel(x1, x0)


def test_gmres_keeps_the_plain_form_where_pivots_are_ill_conditioned(ctx, monkeypatch):
    """p = 3 Euler stage matrices have pivot blocks with cond ~ 1e7 - 1e9, so
    at tolerance 1e-10 the solve runs the plain product: bit for bit the
    result of a preconditioner without the split form."""
    _, _, _, J = newton_system(ctx, "euler", 3)
    plain, split = pair(J, monkeypatch)
    tol = 1e-10
    assert 0.25 * EPS * split.pivot_cond() > tol
    b = rhs(J)
    x0, x1 = torch.zeros_like(b), torch.zeros_like(b)
    r0 = J.gmres(b, x0, 30, tol, 9000, plain)
    r1 = J.gmres(b, x1, 30, tol, 9000, split)
    assert r0 == r1 and torch.equal(x0, x1)


def test_split_not_used_once_the_matrix_changes(ctx, monkeypatch):
    """A factorisation applied to a matrix whose values have changed since
    (a lagged preconditioner) takes the plain product: the result is the
    plain form's bit for bit.  After a refactorisation the split form is
    used again."""
    eq, u, dt, J = newton_system(ctx, "advection", 2)
    plain, split = pair(J, monkeypatch)
    assert split.split_ready(J)
    eq.jacobian(u, 0.0, scale=-2 * dt * GAMMA_SDIRK, add_mass=True, out=J)  # new values, same matrix
    assert not split.split_ready(J)
    b = rhs(J)
    y0 = plain.apply_op(J, b)
    assert torch.equal(split.apply_op(J, b, accuracy=1.0), y0)
    # another matrix with the factorisation's values is not the source either
    J2 = eq.jacobian(u, 0.0, scale=-2 * dt * GAMMA_SDIRK, add_mass=True)
    plain.refactor(J2)
    split.refactor(J)
    assert split.split_ready(J) and not split.split_ready(J2)
    y0 = plain.apply_op(J2, b)
    assert torch.equal(split.apply_op(J2, b, accuracy=1.0), y0)
    # refactored from J's current values: split again
    y2 = split.apply_op(J, b, accuracy=1.0)
    assert not torch.equal(y2, y0)
    assert rel(y2, y0) < 0.25 * EPS * split.pivot_cond()
