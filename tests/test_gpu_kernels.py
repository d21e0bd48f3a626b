"""Kernel-level parity of the CUDA path against the oracle (FP64 unless stated).

Tolerances: 1e-12 relative (max-abs difference over max-abs of the oracle)
for residual, Jacobian, mass, norms and projection -- the two sides sum the
same quadrature terms in different orders; 1e-6 for FP32-stored blocks.
"""
import numpy as np
import pytest

import cpolyg_b200 as cp
import oracle
from cases import equations, mesh, rel, to_dev, to_np

pytestmark = pytest.mark.gpu

TOL = 1e-12

CASES = [("adv_const", 1), ("adv_const", 2), ("adv_const", 3), ("adv_rot", 2), ("euler", 1), ("euler", 2),
         ("euler", 3)]


@pytest.mark.parametrize("name,deg", CASES)
@pytest.mark.parametrize("periodic", [True, False])
def test_residual(ctx, name, deg, periodic):
    ge, oe, _ = equations(ctx, name, deg, n=300, periodic=periodic)
    kind, params = (cp.INIT_VORTEX, [5.0, 0.5, 0.5, 1, 1, 1.4, 1, 1]) if name == "euler" else \
        (cp.INIT_GAUSSIAN, [30.0, 0.4, 0.6])
    u = oe.interp(kind, params)
    b_or = oe.assemble(u, 0.1)
    b_gpu = to_np(ge.assemble(to_dev(u).reshape(ge.np, ge.nc, ge.nb), 0.1))
    assert rel(b_gpu, b_or) < TOL


@pytest.mark.parametrize("name,deg", CASES)
@pytest.mark.parametrize("periodic", [True, False])
def test_jacobian(ctx, name, deg, periodic):
    ge, oe, arrays = equations(ctx, name, deg, n=200, periodic=periodic)
    rng = np.random.default_rng(3)
    kind, params = (cp.INIT_VORTEX, [5.0, 0.5, 0.5, 1, 1, 1.4, 1, 1]) if name == "euler" else \
        (cp.INIT_GAUSSIAN, [30.0, 0.4, 0.6])
    u = oe.interp(kind, params)
    if name == "euler":  # jumps between cells so both Rusanov branches occur
        u = u * (1 + 0.02 * rng.standard_normal(u.size))
    rp, cl, blk = oe.jacobian(u, 0.2)
    J = ge.jacobian(to_dev(u).reshape(ge.np, ge.nc, ge.nb), 0.2)
    grp, gcl, gblk = J.export()
    assert np.array_equal(grp, rp) and np.array_equal(gcl, cl)
    assert rel(gblk, blk) < TOL
    # fused Newton matrix B = scale*J + M  (BlockMatrix::operator*=, Jacobian::operator+=)
    scale = -0.05 * 0.4358
    J2 = ge.jacobian(to_dev(u).reshape(ge.np, ge.nc, ge.nb), 0.2, scale=scale, add_mass=True)
    _, _, b2 = J2.export()
    ref = blk * scale
    M = oe.mass_blocks()
    for i in range(ge.np):
        ref[rp[i]] += M[i]  # both stored [col][row]
    assert rel(b2, ref) < TOL
    # FP32 storage
    J3 = ge.jacobian(to_dev(u).reshape(ge.np, ge.nc, ge.nb), 0.2, precision=cp.F32)
    _, _, b3 = J3.export()
    assert rel(b3, blk) < 1e-6


@pytest.mark.parametrize("deg", [2, 3])
def test_jacobian_exact_mode(ctx, deg):
    """Exact Euler Jacobian (A_x entry fixed, neighbour-state derivatives)."""
    ge, oe, _ = equations(ctx, "euler", deg, n=200, periodic=True, exact_jacobian=True)
    u = oe.interp(cp.INIT_VORTEX, [5.0, 0.5, 0.5, 1, 1, 1.4, 1, 1])
    rp, cl, blk = oe.jacobian(u, 0.0)
    J = ge.jacobian(to_dev(u).reshape(ge.np, ge.nc, ge.nb), 0.0)
    _, _, gblk = J.export()
    assert rel(gblk, blk) < TOL


@pytest.mark.parametrize("name,deg", [("adv_const", 2), ("euler", 3)])
def test_mass_norm_interp(ctx, name, deg):
    ge, oe, _ = equations(ctx, name, deg, n=300, periodic=True)
    kind, params = (cp.INIT_VORTEX, [5.0, 0.5, 0.5, 1, 1, 1.4, 1, 1]) if name == "euler" else \
        (cp.INIT_GAUSSIAN, [30.0, 0.4, 0.6])
    u_or = oe.interp(kind, params, 0.3)
    u_gpu = ge.interp(kind, params, 0.3)
    assert rel(to_np(u_gpu), u_or) < TOL
    # mass blocks: the oracle stores the reference's bl x bl replicated form
    Mo = oe.mass_blocks()
    Mg = ge.mass_blocks()  # [cell][j][k] = M(k, j)
    nb = ge.nb
    assert rel(Mg, Mo[:, :nb, :nb]) < TOL
    x = np.random.default_rng(0).standard_normal(oe.ndof)
    xd = to_dev(x).reshape(ge.np, ge.nc, ge.nb)
    assert rel(to_np(ge.mass_matvec(xd)), oe.mass_matvec(x)) < TOL
    assert rel(to_np(ge.mass_solve(xd)), oe.mass_solve(x)) < 1e-11
    # L2 norm: oracle integrates u^2 by quadrature, the GPU forms u^T M u
    assert rel(ge.L2Norm(u_gpu), oe.l2norm(u_or)) < TOL


@pytest.mark.parametrize("name,deg,kind,params,t", [
    ("adv_const", 2, cp.INIT_GAUSSIAN, [30.0, 0.4, 0.6, 1.0, 1.0, 1.0, 1.0], 0.35),
    ("adv_const", 3, cp.INIT_GAUSSIAN, [30.0, 0.4, 0.6], 0.0),
    ("euler", 3, cp.INIT_VORTEX, [5.0, 0.5, 0.5, 1, 1, 1.4, 1, 1], 0.3),
    ("euler", 2, cp.INIT_DENSITY_BUMP, [0.1, 0.2, 0.5, 0.5, 0.3, 1.4], 0.0)])
def test_l2_error(ctx, name, deg, kind, params, t):
    """MeshFn::L2Error against the oracle's quadrature over the same points,
    for a perturbed field and for the interpolant itself (<= 1e-12 relative
    to the norm of the exact field, which bounds the rounding of the sum)."""
    ge, oe, _ = equations(ctx, name, deg, n=300, periodic=True)
    u_or = oe.interp(kind, params, t)
    u_or = u_or + 0.01 * np.random.default_rng(1).standard_normal(u_or.size)
    scale = np.linalg.norm(oe.l2error(np.zeros_like(u_or), kind, params, t))
    eo = oe.l2error(u_or, kind, params, t)
    eg = ge.L2Error(to_dev(u_or).reshape(ge.np, ge.nc, ge.nb), kind, params, t)
    assert np.abs(eg - eo).max() < 1e-12 * scale
    ui = ge.interp(kind, params, t)
    assert np.abs(ge.L2Error(ui, kind, params, t) - oe.l2error(to_np(ui), kind, params, t)).max() < 1e-12 * scale


def test_field_and_matrix_gnuplot_files(ctx, tmp_path):
    """MeshFn::gnuplot: one line per point of the 3-point rule on every
    sub-triangle, values (evaluated on the device) equal to the oracle's
    Leg2D at those points; BlockMatrix::spy: every entry above 1e-10."""
    ge, oe, a = equations(ctx, "euler", 2, n=120, periodic=True, width=10.0)
    u = oe.interp(cp.INIT_VORTEX, [5.0, 5.0, 5.0, 1, 1, 1.4, 10, 10])
    ud = to_dev(u).reshape(ge.np, ge.nc, ge.nb)
    path = tmp_path / "u.gnu"
    ge.gnuplot(ud, str(path))
    rows = np.array([[float(v) for v in ln.split("\t")] for ln in path.read_text().splitlines()])
    tri = a["tri_xy"].reshape(-1, 6)
    q = np.array([[1 / 6, 1 / 6], [1 / 6, 2 / 3], [2 / 3, 1 / 6]])  # the 3-point rule's (a, b)
    assert rows.shape == (3 * len(tri), 2 + ge.nc)
    k = 0
    nb = ge.nb
    for i in range(ge.np):
        x0, y0, w, h = a["bb"][i]
        for t in range(a["tri_ptr"][i], a["tri_ptr"][i + 1]):
            T = tri[t]
            for qa, qb in q:
                x = T[0] * (1 - qa - qb) + T[2] * qa + T[4] * qb
                y = T[1] * (1 - qa - qb) + T[3] * qa + T[5] * qb
                assert abs(rows[k, 0] - x) <= 1e-5 * max(1.0, abs(x)) and abs(rows[k, 1] - y) <= 1e-5 * max(1.0, abs(y))
                for c in range(ge.nc):
                    want = oracle.leg2d(2 * (x - x0) / w - 1, 2 * (y - y0) / h - 1, 3, u[i * ge.bl + c * nb:][:nb])
                    assert abs(rows[k, 2 + c] - want) <= 1e-12 * max(1.0, abs(want))
                k += 1
    # spy of the Jacobian
    J = ge.jacobian(ud)
    rp, cl, blk = J.export()
    J.spy(str(tmp_path / "J.spy"))
    got = np.loadtxt(tmp_path / "J.spy")
    bl = ge.bl
    want = [(i * bl + ii, cl[k] * bl + jj, blk[k][jj, ii]) for i in range(len(rp) - 1) for k in range(rp[i], rp[i + 1])
            for ii in range(bl) for jj in range(bl) if abs(blk[k][jj, ii]) > 1e-10]
    assert got.shape == (len(want), 3)
    w = np.array(want)
    assert np.array_equal(got[:, :2], w[:, :2])
    assert np.allclose(got[:, 2], w[:, 2], rtol=1e-5)


BLS = [1, 3, 4, 6, 7, 10, 12, 24, 40, 48]


def random_bsr(n_rows, bl, seed=0):
    m, arrays, _ = mesh(60, True, 1.0, 2)
    rp, cl = m.pattern()
    rng = np.random.default_rng(seed + bl)
    blocks = rng.standard_normal((len(cl), bl, bl))
    for i in range(len(rp) - 1):  # diagonally dominant diagonal blocks
        blocks[rp[i]] += np.eye(bl) * (3.0 * bl)
    return rp, cl, blocks


@pytest.mark.parametrize("bl", BLS)
@pytest.mark.parametrize("prec", [cp.F64, cp.F32])
def test_matvec(ctx, bl, prec):
    rp, cl, blocks = random_bsr(60, bl)
    A = cp.BlockMatrix.from_host(ctx, rp, cl, blocks, precision=prec)
    x = np.random.default_rng(1).standard_normal((len(rp) - 1) * bl)
    y = to_np(A.matvec(to_dev(x)))
    ref = oracle.bsr_matvec(rp, cl, blocks.astype(np.float32).astype(np.float64) if prec == cp.F32 else blocks, x)
    assert rel(y, ref) < (1e-13 if prec == cp.F64 else 1e-13)


@pytest.mark.parametrize("bl", [3, 6, 10, 12, 16, 24, 40, 48])
def test_ilu0_factor_apply_and_levels(ctx, bl):
    rp, cl, blocks = random_bsr(60, bl, seed=5)
    A = cp.BlockMatrix.from_host(ctx, rp, cl, blocks)
    P = cp.BlockILU0(A)
    dd, (lr, lc, lb), (ur, uc, ub), sing = oracle.ilu0(rp, cl, blocks)
    assert sing < 0
    gdd, (glr, glc, glb), (gur, guc, gub) = P.export(len(lc), len(uc))
    assert np.array_equal(glr, lr) and np.array_equal(glc, lc)
    assert np.array_equal(gur, ur) and np.array_equal(guc, uc)
    assert rel(gdd, dd) < 1e-11 and rel(glb, lb) < 1e-11 and rel(gub, ub) < 1e-11
    # level schedule: device object, host function and oracle agree byte for byte
    olv = oracle.levels(rp, cl)
    for a, b in zip(P.levels(), olv):
        assert np.array_equal(a, b)
    for a, b in zip(cp.pattern_levels(rp, cl), olv):
        assert np.array_equal(a, b)
    x = np.random.default_rng(2).standard_normal((len(rp) - 1) * bl)
    xd = to_dev(x)
    P.solve(xd)
    assert rel(to_np(xd), oracle.precond_apply(2, rp, cl, blocks, x)) < 1e-11


@pytest.mark.parametrize("bl", [6, 40])
def test_block_jacobi(ctx, bl):
    rp, cl, blocks = random_bsr(60, bl, seed=7)
    A = cp.BlockMatrix.from_host(ctx, rp, cl, blocks)
    P = cp.BlockJacobi(A)
    x = np.random.default_rng(3).standard_normal((len(rp) - 1) * bl)
    xd = to_dev(x)
    P.solve(xd)
    assert rel(to_np(xd), oracle.precond_apply(1, rp, cl, blocks, x)) < 1e-11
    # BlockMatrix::jacobi iteration
    b = np.random.default_rng(4).standard_normal(x.size)
    xo, its_o, res_o = oracle.jacobi(rp, cl, blocks, b, np.zeros_like(b), 1e-10, 500)
    xg = to_dev(np.zeros_like(b))
    its_g, res_g = A.jacobi(to_dev(b), xg, 1e-10, 500, P)
    assert abs(its_g - its_o) <= 1
    assert rel(to_np(xg), xo) < 1e-9


@pytest.mark.parametrize("pc", [cp.PC_NONE, cp.PC_BJACOBI, cp.PC_ILU0])
def test_gmres_vs_oracle(ctx, pc):
    bl = 10
    rp, cl, blocks = random_bsr(60, bl, seed=11)
    A = cp.BlockMatrix.from_host(ctx, rp, cl, blocks)
    P = {cp.PC_NONE: None, cp.PC_BJACOBI: cp.BlockJacobi, cp.PC_ILU0: cp.BlockILU0}[pc]
    P = P(A) if P else None
    b = np.random.default_rng(5).standard_normal((len(rp) - 1) * bl)
    xo, its_o, tol_o = oracle.gmres(pc, rp, cl, blocks, b, np.zeros_like(b), 20, 1e-12, 2000)
    xg = to_dev(np.zeros_like(b))
    its_g, tol_g = A.gmres(to_dev(b), xg, 20, 1e-12, 2000, P)
    assert abs(its_g - its_o) <= 1
    assert rel(to_np(xg), xo) < 1e-10
    dense = np.zeros((b.size, b.size))
    for i in range(len(rp) - 1):
        for k in range(rp[i], rp[i + 1]):
            dense[i * bl:(i + 1) * bl, cl[k] * bl:(cl[k] + 1) * bl] = blocks[k].T
    assert np.linalg.norm(dense @ to_np(xg) - b) < 1e-9 * np.linalg.norm(b)


@pytest.mark.parametrize("mode,tol", [("3", 2e-6), ("1", 2e-3), ("0", 1e-6)])
def test_fp32_ilu_factor_tensor_core_products(ctx, monkeypatch, mode, tol):
    """FP32 factors of 40x40 blocks: the block products run on tcgen05
    kind::tf32 MMAs (mode 3: three TF32 passes, about FP32 accuracy; mode 1:
    one pass) or on FP64 DMMA (mode 0).  Factors and one application against
    the oracle's FP64 factorisation; pivots stay FP64."""
    monkeypatch.setenv("CPG_FACTOR_TC", mode)
    bl = 40
    rp, cl, blocks = random_bsr(60, bl, seed=21)
    A32 = cp.BlockMatrix.from_host(ctx, rp, cl, blocks, precision=cp.F32)
    P = cp.BlockILU0(A32, precision=cp.F32)
    b32 = blocks.astype(np.float32).astype(np.float64)  # the FP32 matrix the GPU sees
    dd, (lr, lc, lb), (ur, uc, ub), sing = oracle.ilu0(rp, cl, b32)
    gdd, (glr, glc, glb), (gur, guc, gub) = P.export(len(lc), len(uc))
    assert rel(glb, lb) < tol and rel(gub, ub) < tol and rel(gdd, dd) < tol
    x = np.random.default_rng(3).standard_normal((len(rp) - 1) * bl)
    xd = to_dev(x)
    P.solve(xd)
    assert rel(to_np(xd), oracle.precond_apply(2, rp, cl, b32, x)) < 10 * tol


def test_fgmres_solves(ctx):
    bl = 40
    rp, cl, blocks = random_bsr(60, bl, seed=13)
    A = cp.BlockMatrix.from_host(ctx, rp, cl, blocks)
    A32 = cp.BlockMatrix.from_host(ctx, rp, cl, blocks, precision=cp.F32)
    P = cp.BlockILU0(A32, precision=cp.F32)
    b = np.random.default_rng(6).standard_normal((len(rp) - 1) * bl)
    xg = to_dev(np.zeros_like(b))
    its, res = A.gmres(to_dev(b), xg, 30, 1e-12, 600, P, flexible=True)
    xo, _, _ = oracle.gmres(2, rp, cl, blocks, b, np.zeros_like(b), 30, 1e-13, 2000)
    assert res < 1e-12
    assert rel(to_np(xg), xo) < 1e-10


def test_singular_pivot_reported(ctx):
    rp, cl, blocks = random_bsr(60, 6, seed=17)
    blocks[rp[5]] = 0.0  # plant a zero diagonal block in a host-built matrix
    for k in range(rp[5], rp[6]):
        blocks[k] = 0.0
    A = cp.BlockMatrix.from_host(ctx, rp, cl, blocks)
    with pytest.raises(cp.CpgError) as e:
        cp.BlockJacobi(A)
    assert e.value.status == 3  # CPG_ERR_SINGULAR_BLOCK
