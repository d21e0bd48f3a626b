"""Batched GMRES: independent systems stacked block-diagonally and solved in
one launch sequence, each with its own Krylov scalars and stopping test
(segmented reductions, Givens rotations on the device).

Each system's reductions run on the same fixed grid as a solve of that
system alone, and its rows are computed row by row, so with the same
triangular-sweep form and matvec variant the batched iterates equal the
single solves' bit for bit: the same iteration counts and the same
solutions."""
import numpy as np
import pytest
import torch

import cpolyg_b200 as cp
import oracle
from cases import rel, to_dev, to_np

pytestmark = pytest.mark.gpu

V = [5.0, 5.0, 5.0, 1.0, 1.0, 1.4, 10.0, 10.0]


def newton_matrices(ctx, sizes, degree=3, precision=cp.F64):
    out = []
    for k, n in enumerate(sizes):
        m = cp.PolyMesh.voronoi(cp.uniform_seeds(10 + k, n, 10.0, 10.0), 10.0, 10.0, periodic=True)
        eq = cp.Euler(ctx, m, degree, dirichlet=(cp.INIT_VORTEX, V), exact_jacobian=True)
        u = eq.interp(cp.INIT_VORTEX, V)
        dt = 0.05 * (100000 / n) ** 0.5
        out.append((eq, eq.jacobian(u, 0.0, scale=-dt * 0.435866521508459, add_mass=True, precision=precision)))
    return out


@pytest.mark.parametrize("flexible,precision", [(False, cp.F64), (True, cp.F32)])
def test_batched_gmres_equals_single_solves(ctx, monkeypatch, flexible, precision):
    # the same triangular-sweep form alone and stacked, and every system
    # large enough (>= 2048 block rows) for the tuned matvec variant
    monkeypatch.setenv("CPG_ILU_SWEEP", "form4")
    sizes = [2100, 2600, 3300, 4100]
    mats = newton_matrices(ctx, sizes, precision=precision)
    Js = [J for _, J in mats]
    gen = torch.Generator("cuda").manual_seed(3)
    bs = [torch.randn(J.n_rows * J.bl, dtype=torch.float64, device="cuda", generator=gen) for J in Js]
    singles = []
    for J, b in zip(Js, bs):
        P = cp.BlockILU0(J, precision=precision)
        x = torch.zeros_like(b)
        its, res = J.gmres(b, x, 30, 1e-10, 9000, P, flexible=flexible)
        singles.append((its, res, x))
    S = cp.BlockMatrix.stack(Js)
    assert list(S.seg_rows) == list(np.cumsum([0] + sizes))
    PS = cp.BlockILU0(S, precision=precision)
    b = torch.cat(bs)
    x = torch.zeros_like(b)
    out = S.gmres_batched(S.seg_rows, b, x, 30, 1e-10, 9000, PS, flexible=flexible)
    bl = Js[0].bl
    for k, ((its, res, xs), (itb, resb)) in enumerate(zip(singles, out)):
        assert its == itb and res == resb and res < 1e-10
        assert torch.equal(x[S.seg_rows[k] * bl:S.seg_rows[k + 1] * bl], xs)


def test_batched_gmres_matches_oracle_per_system(ctx):
    """Systems of different sizes against the oracle's GMRES (the reference's
    algorithm): iteration counts within one, solutions within 1e-10."""
    mats = newton_matrices(ctx, [150, 400], degree=2)
    Js = [J for _, J in mats]
    rng = np.random.default_rng(4)
    bs = [rng.standard_normal(J.n_rows * J.bl) for J in Js]
    S = cp.BlockMatrix.stack(Js)
    P = cp.BlockILU0(S)
    x = to_dev(np.zeros(S.n_rows * S.bl))
    out = S.gmres_batched(S.seg_rows, to_dev(np.concatenate(bs)), x, 30, 1e-12, 3000, P)
    xg = to_np(x)
    bl = S.bl
    for k, (J, b) in enumerate(zip(Js, bs)):
        rp, cl, blk = J.export()
        xo, its_o, _ = oracle.gmres(2, rp, cl, blk, b, np.zeros_like(b), 30, 1e-12, 3000)
        assert abs(out[k][0] - its_o) <= 1
        assert rel(xg[S.seg_rows[k] * bl:S.seg_rows[k + 1] * bl], xo) < 1e-10


def test_batched_gmres_rejects_coupled_systems(ctx):
    mats = newton_matrices(ctx, [150], degree=1)
    J = mats[0][1]
    half = J.n_rows // 2
    b = torch.zeros(J.n_rows * J.bl, dtype=torch.float64, device="cuda")
    with pytest.raises(cp.CpgError) as e:
        J.gmres_batched([0, half, J.n_rows], b, b.clone(), 10, 1e-8, 100)
    assert e.value.status == 1 and "couples two systems" in str(e.value)


def advection_matrices(ctx, sizes, degree=2):
    out = []
    for k, n in enumerate(sizes):
        m = cp.PolyMesh.voronoi(cp.uniform_seeds(30 + k, n, 1.0, 1.0), 1.0, 1.0, periodic=True)
        eq = cp.ConstantAdvection(ctx, m, degree, 1.0, 0.5)
        u = eq.interp(cp.INIT_GAUSSIAN, [100.0, 0.5, 0.5])
        out.append(eq.jacobian(u, 0.0, scale=-0.05 * 0.435866521508459, add_mass=True))
    return out


def test_batched_gmres_equals_single_solves_in_split_form(ctx, monkeypatch):
    """Well-conditioned pivot blocks (p = 2 advection): every solve takes the
    split form of P^{-1} A, and the batched iterates still equal the single
    solves' bit for bit (E and the split rows are row-local)."""
    monkeypatch.setenv("CPG_ILU_SWEEP", "form4")
    tol = 1e-10
    Js = advection_matrices(ctx, [2100, 2600, 3300])
    gen = torch.Generator("cuda").manual_seed(8)
    bs = [torch.randn(J.n_rows * J.bl, dtype=torch.float64, device="cuda", generator=gen) for J in Js]
    singles = []
    for J, b in zip(Js, bs):
        P = cp.BlockILU0(J)
        assert P.split_ready(J) and 0.25 * 2.0 ** -52 * P.pivot_cond() <= tol
        x = torch.zeros_like(b)
        its, res = J.gmres(b, x, 30, tol, 9000, P)
        singles.append((its, res, x))
    S = cp.BlockMatrix.stack(Js)
    PS = cp.BlockILU0(S)
    assert PS.split_ready(S) and 0.25 * 2.0 ** -52 * PS.pivot_cond() <= tol
    x = torch.zeros(S.n_rows * S.bl, dtype=torch.float64, device="cuda")
    out = S.gmres_batched(S.seg_rows, torch.cat(bs), x, 30, tol, 9000, PS)
    bl = S.bl
    for k, ((its, res, xs), (itb, resb)) in enumerate(zip(singles, out)):
        assert its == itb and res == resb and res < tol
        assert torch.equal(x[S.seg_rows[k] * bl:S.seg_rows[k + 1] * bl], xs)
