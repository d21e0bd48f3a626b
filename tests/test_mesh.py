"""Host mesh: Voronoi construction, connectivity and the block pattern /
ILU(0) level schedule, checked byte for byte against the oracle's own
derivation (PolyMesh::computep2p / computebb / getOutwardNormal semantics)."""
import numpy as np
import pytest

import cpolyg_b200 as cp
import oracle
from cases import mesh


def polygon_areas(a):
    cp_, xy = a["cell_ptr"], a["poly_xy"]
    out = []
    for i in range(len(cp_) - 1):
        p = xy[cp_[i]:cp_[i + 1]]
        x, y = p[:, 0], p[:, 1]
        out.append(0.5 * np.sum(x * np.roll(y, -1) - np.roll(x, -1) * y))
    return np.array(out)


@pytest.mark.parametrize("n,periodic,width", [(1000, True, 1.0), (1000, False, 1.0), (3000, True, 10.0),
                                              (2000, False, 10.0)])
def test_voronoi_tiles_domain(n, periodic, width):
    m, a, om = mesh(n, periodic, width)
    areas = polygon_areas(a)
    assert (areas > 0).all()  # counter-clockwise convex cells
    assert abs(areas.sum() - width * width) < 1e-10 * width * width
    # each cell contains its seed
    seeds = cp.uniform_seeds(1, n, width, width)
    assert np.allclose(a["bb"][:, 0] <= seeds[:, 0], True)
    # p2p symmetric; periodic shifts are opposite
    nbr, cptr, sh = a["edge_nbr"], a["cell_ptr"], a["edge_shift"]
    for i in range(n):
        for e in range(cptr[i], cptr[i + 1]):
            j = nbr[e]
            if j < 0:
                assert not periodic
                continue
            back = [f for f in range(cptr[j], cptr[j + 1]) if nbr[f] == i]
            assert len(back) == 1
            assert np.array_equal(sh[back[0]], -sh[e])
    avg = len(nbr) / n
    assert 5.5 < avg < 6.5


@pytest.mark.parametrize("n,periodic,width", [(1000, True, 1.0), (1000, False, 1.0), (5000, True, 10.0)])
def test_connectivity_matches_oracle(n, periodic, width):
    m, a, om = mesh(n, periodic, width)
    o = om.export()
    assert np.array_equal(o["cell_ptr"], a["cell_ptr"])
    assert np.array_equal(o["edge_nbr"], a["edge_nbr"])
    assert np.array_equal(o["edge_shift"], a["edge_shift"])
    assert np.array_equal(o["bb"], a["bb"])
    # block pattern (Jacobian ctor) and level schedule, byte-equal
    rp, cl = m.pattern()
    oe = oracle.Equation(om, 0, 1)
    orp, ocl, _ = oe.jacobian(np.zeros(oe.ndof))
    assert np.array_equal(rp, orp) and np.array_equal(cl, ocl)
    for x, y in zip(cp.pattern_levels(rp, cl), oracle.levels(rp, cl)):
        assert np.array_equal(x, y)


def test_box_boundary_codes():
    codes = (cp.BC_WALL, cp.BC_OUTFLOW, cp.BC_WALL, cp.BC_INFLOW)
    m, a, om = mesh(500, False, 10.0, 5, codes)
    nbr, xy, cptr = a["edge_nbr"], a["poly_xy"], a["cell_ptr"]
    seen = set()
    for i in range(len(cptr) - 1):
        s, e = cptr[i], cptr[i + 1]
        for k in range(s, e):
            if nbr[k] >= 0:
                continue
            p, q = xy[k], xy[s + (k - s + 1) % (e - s)]
            mid = 0.5 * (p + q)
            if abs(mid[1]) < 1e-9 or abs(mid[1] - 10) < 1e-9:
                assert nbr[k] == cp.BC_WALL
            elif abs(mid[0] - 10) < 1e-9:
                assert nbr[k] == cp.BC_OUTFLOW
            else:
                assert abs(mid[0]) < 1e-9 and nbr[k] == cp.BC_INFLOW
            seen.add(int(nbr[k]))
    assert seen == {cp.BC_WALL, cp.BC_OUTFLOW, cp.BC_INFLOW}
    assert np.array_equal(om.export()["edge_nbr"], nbr)


def test_large_mesh_levels_are_few():
    """Random (seed) order gives a short level schedule for ILU(0)."""
    m, a, om = mesh(20000, True, 10.0, 2)
    rp, cl = m.pattern()
    lp, lr, up, ur = cp.pattern_levels(rp, cl)
    assert len(lp) - 1 < 40 and len(up) - 1 < 40
    assert sorted(lr.tolist()) == list(range(20000))


def test_quad_mesh_from_polygons():
    polys = []
    N = 4
    for j in range(N):
        for i in range(N):
            x0, y0 = i / N, j / N
            polys.append([(x0, y0), (x0 + 1 / N, y0), (x0 + 1 / N, y0 + 1 / N), (x0, y0 + 1 / N)])
    m = cp.PolyMesh.from_polygons(polys, 1.0, 1.0, periodic=True)
    a = m.export()
    assert a["edge_nbr"].min() >= 0 and len(a["edge_nbr"]) == 4 * N * N
    # coarse periodic meshes whose cells meet twice are rejected
    with pytest.raises(cp.CpgError):
        cp.PolyMesh.voronoi(cp.uniform_seeds(3, 3), 1, 1, periodic=True)


def _rotate_to_match(P, Q):
    """rotation of the cyclic vertex list Q that best matches P (max abs diff)"""
    best = None
    for r in range(len(Q)):
        d = np.abs(np.roll(Q, -r, axis=0) - P).max()
        best = d if best is None else min(best, d)
    return best


@pytest.mark.parametrize("n,periodic,width,seed", [(2000, True, 10.0, 2), (1500, False, 1.0, 1)])
def test_voronoi_cells_match_brute_force_oracle(n, periodic, width, seed):
    """The library's bucket-grid mesher against the oracle's brute-force
    half-plane clipping of the same seeds: same polygons vertex for vertex
    (up to the start vertex, within 1e-9 of the domain size) and the same
    neighbour set of every cell, periodic and not."""
    seeds = cp.uniform_seeds(seed, n, width, width)
    assert np.array_equal(seeds, oracle.uniform_seeds(seed, n, width, width))
    m = cp.PolyMesh.voronoi(seeds, width, width, periodic=periodic)
    a = m.export()
    om = oracle.Mesh.voronoi(seeds, width, width, periodic=periodic)
    ocp, oxy = om.polygons()
    onbr = om.export()["edge_nbr"]
    assert np.array_equal(np.diff(ocp), np.diff(a["cell_ptr"]))
    for i in range(n):
        P = a["poly_xy"][a["cell_ptr"][i]:a["cell_ptr"][i + 1]]
        Q = oxy[ocp[i]:ocp[i + 1]]
        assert _rotate_to_match(P, Q) < 1e-9 * width
        assert set(a["edge_nbr"][a["cell_ptr"][i]:a["cell_ptr"][i + 1]]) == set(onbr[ocp[i]:ocp[i + 1]])


def test_benchmark_mesh_pattern_and_levels_match_oracle():
    """The 100k-cell periodic benchmark mesh (seed 2, [0,10]^2): edge
    neighbours, periodic shifts, bounding boxes, the Jacobian block pattern
    (Jacobian ctor, src/Jacobian.cpp:7-47) and the ILU(0) level schedule
    (the dependency order of src/Preconditioners.cpp:49-158), derived by the
    oracle from the cell polygons alone, byte for byte."""
    seeds = cp.uniform_seeds(2, 100000, 10.0, 10.0)
    m = cp.PolyMesh.voronoi(seeds, 10.0, 10.0, periodic=True)
    a = m.export()
    om = oracle.Mesh(a)
    o = om.export()
    for k in ("cell_ptr", "edge_nbr", "edge_shift", "bb"):
        assert np.array_equal(o[k], a[k]), k
    rp, cl = m.pattern()
    orp, ocl = om.pattern()
    assert np.array_equal(rp, orp) and np.array_equal(cl, ocl)
    assert len(cl) == 100000 + len(a["edge_nbr"])
    for x, y in zip(cp.pattern_levels(rp, cl), oracle.levels(rp, cl)):
        assert np.array_equal(x, y)


def test_mesh_gnuplot_file(tmp_path):
    """PolyMesh::gnuplot format: "# polygon number i", the vertices with the
    first one repeated, a blank line; the cell's own frame."""
    m, a, _ = mesh(300, True, 1.0)
    path = tmp_path / "edges.gnu"
    m.gnuplot(str(path))
    blocks = path.read_text().strip("\n").split("\n\n")
    assert len(blocks) == 300
    for i, b in enumerate(blocks):
        lines = b.split("\n")
        assert lines[0] == f"# polygon number {i}"
        pts = np.array([[float(v) for v in ln.split("\t")] for ln in lines[1:]])
        P = a["poly_xy"][a["cell_ptr"][i]:a["cell_ptr"][i + 1]]
        assert len(pts) == len(P) + 1 and np.array_equal(pts[0], pts[-1])
        assert np.allclose(pts[:-1], P, rtol=1e-5, atol=1e-6)
