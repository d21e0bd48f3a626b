"""Serving loop: admission by HBM footprint, overlap of requests in flight,
and per-request results that are the same alone and in the mix."""
import math

import numpy as np
import pytest

from cpolyg_b200 import serve


def test_stream_mix_and_footprints():
    reqs = serve.make_stream(512, rate=200.0, seed=0)
    assert len(reqs) == 512
    adv = [r for r in reqs if r.physics == "advection"]
    eul = [r for r in reqs if r.physics == "euler"]
    assert 0.4 < len(adv) / 512 < 0.6
    assert {r.degree for r in adv} == {1, 2, 3} and {r.degree for r in eul} == {2, 3}
    assert all(1 <= r.strength <= 5 for r in eul)
    assert all(0 <= r.angle < 2 * math.pi for r in adv)
    sizes = np.array([r.n_seeds for r in reqs])
    assert sizes.min() >= 500 and sizes.max() <= 50000
    # log-uniform: the median sits near the geometric mean of the range
    assert 2500 < np.median(sizes) < 10000
    gaps = np.diff([r.arrival for r in reqs])
    assert (gaps > 0).all() and 0.003 < gaps.mean() < 0.007  # 200 / s
    steppers = [r.stepper for r in reqs]
    assert 0.4 < steppers.count("rk4") / 512 < 0.6
    assert all(10 <= r.steps <= 100 for r in reqs)
    # implicit requests hold the Jacobian and ILU factors: larger footprint
    a = serve.Request(0, "euler", 3, 10000, 1, "dirk3", 10, 0.01)
    b = serve.Request(0, "euler", 3, 10000, 1, "rk4", 10, 0.01)
    assert serve.footprint(a) > 10 * serve.footprint(b)
    assert serve.footprint(a) > 2 * 7 * 10000 * 40 * 40 * 8


def small_stream():
    reqs = serve.make_stream(10, rate=400.0, seed=3, min_seeds=300, max_seeds=2000, min_steps=3, max_steps=6)
    return reqs


@pytest.mark.gpu
def test_results_identical_alone_and_in_the_mix():
    mix = small_stream()
    srv = serve.Server(slots=4)
    stats = srv.serve(mix, realtime=True)
    assert stats["failed"] == 0 and stats["solves"] == len(mix)
    assert srv.peak_active > 1  # requests overlapped on the device
    for r in mix:
        alone = serve.Request(**{k: getattr(r, k) for k in ("rid", "physics", "degree", "n_seeds", "seed",
                                                            "stepper", "steps", "dt", "angle", "strength")})
        serve.run_request(alone)
        assert np.array_equal(alone.result, r.result), f"request {r.rid} differs in the mix"


@pytest.mark.gpu
def test_admission_respects_the_memory_budget():
    reqs = small_stream()
    biggest = max(serve.footprint(r) for r in reqs)
    srv = serve.Server(slots=8, hbm_budget=biggest)  # room for one big request at a time
    stats = srv.serve(reqs, realtime=False)
    assert stats["failed"] == 0
    assert srv.peak_bytes <= biggest


@pytest.mark.gpu
def test_served_results_match_the_oracle():
    """A sample of served requests, each against the oracle run of the same
    problem (same seeded mesh, physics, stepper, time step and steps):
    relative 2-norm difference <= 1e-11 (FP64)."""
    import cpolyg_b200 as cp
    import oracle
    reqs = serve.make_stream(8, rate=400.0, seed=11, min_seeds=200, max_seeds=600, min_steps=2, max_steps=4)
    srv = serve.Server(slots=4)
    stats = srv.serve(reqs, realtime=True)
    assert stats["failed"] == 0
    kinds = set()
    for r in reqs:
        L = serve.domain(r)
        m = cp.PolyMesh.voronoi(cp.uniform_seeds(r.seed, r.n_seeds, L, L), L, L, periodic=True)
        om = oracle.Mesh(m.export())
        if r.physics == "advection":
            oe = oracle.Equation(om, 0, r.degree, beta=(math.cos(r.angle), math.sin(r.angle)))
            u = oe.interp(cp.INIT_GAUSSIAN, [100.0, 0.5, 0.5])
        else:
            vort = [r.strength, 5.0, 5.0, 1.0, 1.0, 1.4, 10.0, 10.0]
            oe = oracle.Equation(om, 2, r.degree, dkind=cp.INIT_VORTEX, dparams=vort, exact_jacobian=True)
            u = oe.interp(cp.INIT_VORTEX, vort)
        if r.stepper == "rk4":
            st = oracle.Stepper(oe, cp.STEP_RK4)
        else:
            st = oracle.Stepper(oe, cp.STEP_SDIRK3, pc=2, gmres_m=30, gmres_tol=1e-10, gmres_maxit=90000)
        t = 0.0
        for _ in range(r.steps):
            u = st.advance(u, r.dt, t)
            t += r.dt
        err = np.linalg.norm(r.result - u) / np.linalg.norm(u)
        assert err < 1e-11, (r.rid, r.physics, r.stepper, err)
        kinds.add((r.physics, r.stepper))
    assert len(kinds) >= 3  # the sample covers the mix
