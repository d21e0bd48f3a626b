"""Pins against the reference's own code.

The reference's numerical core needs Armadillo, GSL and LAPACK (absent), so
it cannot be built; its vendored mesh libraries can.  oracle/_ref holds
Voro++ 2D and Triangle compiled from the reference tree plus a driver that
calls them as PolyMesh(pts, w, h) and Triangulation do.  These tests check:
  * this project's Voronoi cells equal the reference's (same vertices, same
    neighbour sets) for the same seeds;
  * quadrature over the reference's Triangle "zQq" sub-triangulation and over
    this project's centroid fans agrees for polynomial integrands (mass
    matrices, the constant-velocity advection residual), so the choice of
    sub-triangulation is invisible at round-off for those.
"""
import ctypes as C
import os

import numpy as np
import pytest

import cpolyg_b200 as cp
import oracle
from cases import mesh

LIB = os.path.join(os.path.dirname(oracle.__file__), "_ref", "libref_mesh.so")
pytestmark = pytest.mark.skipif(not os.path.exists(LIB), reason="reference mesh libraries not built")


def ref_lib():
    lib = C.CDLL(LIB)
    lib.ref_voronoi.restype = C.c_int
    lib.ref_voronoi.argtypes = [C.c_int, C.POINTER(C.c_double), C.c_double, C.c_double, C.POINTER(C.c_int),
                                C.POINTER(C.c_double), C.c_int]
    lib.ref_triangulate.restype = C.c_int
    lib.ref_triangulate.argtypes = [C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_int]
    return lib


def ref_voronoi(seeds, w, h):
    lib = ref_lib()
    n = len(seeds)
    xy = np.ascontiguousarray(seeds, np.float64)
    ptr = np.zeros(n + 1, np.int32)
    cap = 40 * n
    poly = np.zeros((cap, 2))
    got = lib.ref_voronoi(n, oracle.pd(xy), w, h, oracle.pi(ptr), oracle.pd(poly), cap)
    assert got > 0
    return ptr, poly[:got]


def ref_triangulate(pts):
    lib = ref_lib()
    pts = np.ascontiguousarray(pts, np.float64)
    out = np.zeros((200, 6))
    nt = lib.ref_triangulate(len(pts), oracle.pd(pts), oracle.pd(out), 200)
    assert nt > 0
    return out[:nt]


def test_voronoi_cells_match_reference():
    n = 1000
    seeds = cp.uniform_seeds(1, n, 1.0, 1.0)
    rptr, rpoly = ref_voronoi(seeds, 1.0, 1.0)
    m, a, om = mesh(n, False, 1.0, 1)
    ptr, poly = a["cell_ptr"], a["poly_xy"]
    assert np.array_equal(np.diff(rptr), np.diff(ptr))  # same vertex counts
    for i in range(n):
        P = poly[ptr[i]:ptr[i + 1]]
        R = rpoly[rptr[i]:rptr[i + 1]]
        # same vertices up to the starting point (the reference container's
        # walls sit at 1 + 1e-10)
        d = np.abs(P[:, None, :] - R[None, :, :]).sum(-1)
        assert d.min(1).max() < 5e-10 and d.min(0).max() < 5e-10
    # neighbour sets: the oracle's restatement of computep2p on the
    # reference polygons against this project's mesh
    tris = np.zeros((0, 6))
    ref_arrays = dict(cell_ptr=rptr, poly_xy=rpoly, tri_ptr=np.zeros(n + 1, np.int32), tri_xy=tris, width=1.0,
                      height=1.0, periodic=False)
    ro = oracle.Mesh(ref_arrays).export()
    for i in range(n):
        mine = sorted(int(x) for x in a["edge_nbr"][ptr[i]:ptr[i + 1]] if x >= 0)
        ref = sorted(int(x) for x in ro["edge_nbr"][rptr[i]:rptr[i + 1]] if x >= 0)
        assert mine == ref


@pytest.mark.parametrize("p", [1, 2, 3])
def test_subtriangulation_invisible_for_polynomials(p):
    n = 300
    m, a, om = mesh(n, True, 1.0, 1)
    ptr, poly = a["cell_ptr"], a["poly_xy"]
    tri_ptr, tris = [0], []
    for i in range(n):
        T = ref_triangulate(poly[ptr[i]:ptr[i + 1]])
        tris.append(T)
        tri_ptr.append(tri_ptr[-1] + len(T))
    ref_arrays = dict(a)
    ref_arrays["tri_ptr"] = np.array(tri_ptr, np.int32)
    ref_arrays["tri_xy"] = np.concatenate(tris)
    avg = len(ref_arrays["tri_xy"]) / n
    assert 6.0 < avg < 14.0  # Triangle's quality refinement adds Steiner points
    om_ref = oracle.Mesh(ref_arrays)
    e_mine = oracle.Equation(om, 0, p, beta=(1.0, 1.0))
    e_ref = oracle.Equation(om_ref, 0, p, beta=(1.0, 1.0))
    Mm, Mr = e_mine.mass_blocks(), e_ref.mass_blocks()
    # the tables carry 14 digits, so "exact" means ~1e-13 relative
    assert np.abs(Mm - Mr).max() < 1e-12 * np.abs(Mr).max()
    u = np.random.default_rng(p).standard_normal(e_mine.ndof)
    bm, br = e_mine.assemble(u), e_ref.assemble(u)
    assert np.abs(bm - br).max() < 1e-12 * np.abs(br).max()


def _ref_subtriangles(a, n):
    ptr, poly = a["cell_ptr"], a["poly_xy"]
    tri_ptr, tris = [0], []
    for i in range(n):
        T = ref_triangulate(poly[ptr[i]:ptr[i + 1]])
        tris.append(T)
        tri_ptr.append(tri_ptr[-1] + len(T))
    return np.array(tri_ptr, np.int32), np.concatenate(tris)


def test_library_takes_reference_subtriangles():
    """cpg_mesh_set_subtriangles accepts the reference's Triangle "zQq"
    sub-triangulation, exports it back, and rejects triangles that do not
    tile the cells."""
    n = 200
    m = cp.PolyMesh.voronoi(cp.uniform_seeds(4, n, 10.0, 10.0), 10.0, 10.0, periodic=True)
    a = m.export()
    tp, tx = _ref_subtriangles(a, n)
    bad = tx.copy()
    bad[0, 2:4] = 0.5 * (bad[0, 0:2] + bad[0, 2:4])  # halve the first triangle
    with pytest.raises(cp.CpgError):
        m.set_subtriangles(tp, bad)
    m.set_subtriangles(tp, tx)
    b = m.export()
    assert m.n_tris == len(tx)
    assert np.array_equal(b["tri_ptr"], tp) and np.array_equal(b["tri_xy"].reshape(-1, 6), tx)


@pytest.mark.gpu
@pytest.mark.parametrize("deg", [2, 3])
def test_euler_on_reference_subtriangles_matches_oracle(ctx, deg):
    """The Euler residual and Jacobian integrated on the reference's Triangle
    "zQq" sub-triangles (src/Triangulation.cpp:11-101) against the oracle on
    the same triangles, <= 1e-12 relative: with them the library's Euler
    results carry the reference's quadrature, not the centroid fans'."""
    n = 300
    V = [5.0, 5.0, 5.0, 1.0, 1.0, 1.4, 10.0, 10.0]
    m = cp.PolyMesh.voronoi(cp.uniform_seeds(2, n, 10.0, 10.0), 10.0, 10.0, periodic=True)
    a = m.export()
    tp, tx = _ref_subtriangles(a, n)
    m.set_subtriangles(tp, tx)
    arrays = dict(a)
    arrays["tri_ptr"], arrays["tri_xy"] = tp, tx
    oe = oracle.Equation(oracle.Mesh(arrays), 2, deg, dkind=2, dparams=V)
    ge = cp.Euler(ctx, m, deg, dirichlet=(cp.INIT_VORTEX, V))
    u = oe.interp(2, V)
    ud = __import__("torch").as_tensor(u).cuda().reshape(ge.np, ge.nc, ge.nb)
    b_or = oe.assemble(u)
    b_gpu = ge.assemble(ud).cpu().numpy().ravel()
    assert np.abs(b_gpu - b_or).max() < 1e-12 * np.abs(b_or).max()
    rp, cl, blk = oe.jacobian(u)
    _, _, gblk = ge.jacobian(ud).export()
    assert np.abs(gblk - blk).max() < 1e-12 * np.abs(blk).max()
    # the fans give another quadrature of the non-polynomial Euler flux
    oe_fan = oracle.Equation(oracle.Mesh(a), 2, deg, dkind=2, dparams=V)
    assert np.abs(oe_fan.assemble(u) - b_or).max() > 1e-9 * np.abs(b_or).max()
