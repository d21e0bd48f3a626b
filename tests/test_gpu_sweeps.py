"""Triangular sweep forms of the block ILU(0) preconditioner.

The sync-free form (one launch per sweep, rows published through per-row
flags) and the level form (one launch per level) stream the same rows with
the same threads per row and sum in the same order, so their results must be
bitwise identical, and the timed choice between them (the first four
applications alternate) must not change any result.  The bounded waits of
the sync-free form are checked by a sweep whose dependency is never
published: the wait runs out, the solve reports CPG_ERR_TIMEOUT, and the
context stays usable."""
import numpy as np
import pytest
import torch

import cpolyg_b200 as cp
import oracle
from cases import mesh, rel, to_dev, to_np

pytestmark = pytest.mark.gpu


def bsr(n, bl, seed):
    m, _, _ = mesh(n, True, 1.0, 2)
    rp, cl = m.pattern()
    rng = np.random.default_rng(seed)
    blocks = rng.standard_normal((len(cl), bl, bl))
    for i in range(len(rp) - 1):
        blocks[rp[i]] += np.eye(bl) * (3.0 * bl)
    return rp, cl, blocks


@pytest.mark.parametrize("bl", [6, 10, 24, 40])
@pytest.mark.parametrize("prec", [cp.F64, cp.F32])
def test_sweep_forms_are_bitwise_equal(ctx, monkeypatch, bl, prec):
    rp, cl, blocks = bsr(1500, bl, 40 + bl)
    A = cp.BlockMatrix.from_host(ctx, rp, cl, blocks, precision=prec)
    monkeypatch.setenv("CPG_ILU_SWEEP", "syncfree")
    P1 = cp.BlockILU0(A, precision=prec)
    monkeypatch.setenv("CPG_ILU_SWEEP", "levels")
    P2 = cp.BlockILU0(A, precision=prec)
    monkeypatch.setenv("CPG_ILU_SWEEP", "levels_wide")
    P3 = cp.BlockILU0(A, precision=prec)
    monkeypatch.setenv("CPG_ILU_SWEEP", "syncfree_direct")
    P6 = cp.BlockILU0(A, precision=prec)
    monkeypatch.setenv("CPG_ILU_SWEEP", "form5")
    P7 = cp.BlockILU0(A, precision=prec)
    monkeypatch.setenv("CPG_ILU_SWEEP", "form6")
    P8 = cp.BlockILU0(A, precision=prec)
    monkeypatch.delenv("CPG_ILU_SWEEP")
    P4 = cp.BlockILU0(A, precision=prec)
    lib = cp.lib()
    assert [lib.cpg_precond_sweep_form(P.h) for P in (P1, P2, P3, P6, P7, P8)] == [1, 2, 3, 4, 5, 6]
    x = to_dev(np.random.default_rng(bl).standard_normal((len(rp) - 1) * bl))
    y1 = P1.solve(x.clone())
    y2 = P2.solve(x.clone())
    y3 = P3.solve(x.clone())
    y6 = P6.solve(x.clone())
    y7 = P7.solve(x.clone())
    y8 = P8.solve(x.clone())
    # same threads per row: same summation order
    assert torch.equal(y1, y2) and torch.equal(y1, y6)
    for y in (y3, y7, y8):  # other widths: other summation orders
        assert rel(to_np(y), to_np(y1)) < (1e-13 if prec == cp.F64 else 1e-6)
    expected = {1: y1, 2: y1, 3: y3, 4: y1, 5: y7, 6: y8}
    # timed choice (on a scratch copy): the caller only sees the decided form
    y4 = P4.solve(x.clone())
    form = lib.cpg_precond_sweep_form(P4.h)
    assert form in expected
    assert torch.equal(y4, expected[form])
    # the decision holds for the next preconditioner of the same class
    P5 = cp.BlockILU0(A, precision=prec)
    assert lib.cpg_precond_sweep_form(P5.h) == form
    if prec == cp.F64:
        assert rel(to_np(y1), oracle.precond_apply(2, rp, cl, blocks, to_np(x))) < 1e-11


def test_sync_free_sweep_waits_run_out_and_report(ctx):
    lib = cp.lib()
    st = lib.cpg_debug_sweep_timeout(ctx.h)
    assert st == 6, lib.cpg_last_error(ctx.h)  # CPG_ERR_TIMEOUT
    # the context still works, and the status word was cleared
    rp, cl, blocks = bsr(300, 6, 3)
    A = cp.BlockMatrix.from_host(ctx, rp, cl, blocks)
    P = cp.BlockILU0(A)
    x = np.random.default_rng(0).standard_normal((len(rp) - 1) * 6)
    y = to_np(P.solve(to_dev(x)))
    assert rel(y, oracle.precond_apply(2, rp, cl, blocks, x)) < 1e-11


def _forms(ctx, monkeypatch, A, prec, forms):
    out = {}
    for f in forms:
        monkeypatch.setenv("CPG_ILU_SWEEP", f"form{f}")
        out[f] = cp.BlockILU0(A, precision=prec)
        assert cp.lib().cpg_precond_sweep_form(out[f].h) == f
    monkeypatch.delenv("CPG_ILU_SWEEP")
    return out


@pytest.mark.parametrize("prec", [cp.F64, cp.F32])
def test_sweep_forms_at_scale_on_the_newton_matrix(ctx, monkeypatch, prec):
    """20,000 block rows of 40x40 (the p=3 Euler Newton matrix of the vortex
    at the benchmark's dt/h), so the sync-free forms run with many CTAs in
    flight and rows waiting on rows of other CTAs: forms with the same threads
    per row agree bit for bit with the level form, the others within the
    rounding of another summation order."""
    n = 20000
    V = [5.0, 5.0, 5.0, 1.0, 1.0, 1.4, 10.0, 10.0]
    m = cp.PolyMesh.voronoi(cp.uniform_seeds(2, n, 10.0, 10.0), 10.0, 10.0, periodic=True)
    eq = cp.Euler(ctx, m, 3, dirichlet=(cp.INIT_VORTEX, V), exact_jacobian=True)
    u = eq.interp(cp.INIT_VORTEX, V)
    J = eq.jacobian(u, 0.0, scale=-0.05 * (100000 / n) ** 0.5 * 0.435866521508459, add_mass=True, precision=prec)
    P = _forms(ctx, monkeypatch, J, prec, [1, 2, 3, 4, 5, 6])
    x = torch.randn(n * 40, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(7))
    y = {f: p.solve(x.clone()) for f, p in P.items()}
    assert torch.equal(y[1], y[2]) and torch.equal(y[4], y[2])
    for f in (3, 5, 6):
        assert rel(to_np(y[f]), to_np(y[2])) < (1e-12 if prec == cp.F64 else 1e-5)
    # repeated applications reuse the flags with a new generation
    assert torch.equal(P[4].solve(x.clone()), y[4])


def test_sync_free_sweep_at_scale_matches_oracle(ctx, monkeypatch):
    """30,000 block rows of 10x10 against the oracle's BlockILU0 solve."""
    rp, cl, blocks = bsr(30000, 10, 11)
    A = cp.BlockMatrix.from_host(ctx, rp, cl, blocks)
    P = _forms(ctx, monkeypatch, A, cp.F64, [1, 4])
    x = np.random.default_rng(5).standard_normal((len(rp) - 1) * 10)
    want = oracle.precond_apply(2, rp, cl, blocks, x)
    for p in P.values():
        assert rel(to_np(p.solve(to_dev(x))), want) < 1e-11
