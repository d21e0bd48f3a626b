"""Continuous-batching serving loop for independent DG solves.

Requests arrive on their own clock (Poisson arrivals in the benchmark).  A
scheduler admits them in arrival order as soon as a slot and enough device
memory (the request's HBM footprint, estimated from its mesh size, degree,
physics and stepper) are free.  Every admitted request runs on its own
library context and CUDA stream, driven by a worker thread, so the kernels of
requests in flight overlap on the device while new requests keep being
admitted.  Requests never share reductions or buffers, and every reduction
runs on a fixed grid, so a request's result does not depend on what else is
in flight.
"""
from __future__ import annotations

import math
import threading
import time
from dataclasses import dataclass, field

import numpy as np

import cpolyg_b200 as cp

GAMMA = 1.4


@dataclass
class Request:
    rid: int
    physics: str            # "advection" or "euler"
    degree: int
    n_seeds: int
    seed: int
    stepper: str            # "rk4" or "dirk3"
    steps: int
    dt: float
    angle: float = 0.0      # advection velocity angle
    strength: float = 5.0   # vortex strength
    arrival: float = 0.0    # seconds since the stream started
    # filled by the server
    admitted: float = math.nan
    done: float = math.nan
    result: np.ndarray | None = field(default=None, repr=False)
    error: str | None = None
    newton: int = 0
    gmres: int = 0


def make_stream(n: int = 512, rate: float = 200.0, seed: int = 0, min_seeds: int = 500, max_seeds: int = 50000,
                min_steps: int = 10, max_steps: int = 100) -> list[Request]:
    """The serving mix: 50% advection (p in {1,2,3}, velocity angle uniform
    in [0, 2 pi)), 50% Euler vortex (p in {2,3}, strength uniform in [1,5]);
    log-uniform mesh sizes; RK4 or 3-stage DIRK (SDIRK3) 50/50; Poisson
    arrivals."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for rid in range(n):
        t += rng.exponential(1.0 / rate)
        adv = rng.random() < 0.5
        ns = int(round(math.exp(rng.uniform(math.log(min_seeds), math.log(max_seeds)))))
        stepper = "rk4" if rng.random() < 0.5 else "dirk3"
        steps = int(rng.integers(min_steps, max_steps + 1))
        if adv:
            deg = int(rng.choice([1, 2, 3]))
            req = Request(rid, "advection", deg, ns, rid + 1, stepper, steps, 0.0,
                          angle=float(rng.uniform(0, 2 * math.pi)))
        else:
            deg = int(rng.choice([2, 3]))
            req = Request(rid, "euler", deg, ns, rid + 1, stepper, steps, 0.0,
                          strength=float(rng.uniform(1, 5)))
        req.dt = cfl_dt(req)
        req.arrival = t
        out.append(req)
    return out


def domain(req: Request) -> float:
    return 1.0 if req.physics == "advection" else 10.0


def cfl_dt(req: Request) -> float:
    """Time step rule: explicit RK4 at CFL 0.1 of h/((2p+1)|lambda|max),
    DIRK3 at 10x that (h = domain / sqrt(cells))."""
    h = domain(req) / math.sqrt(req.n_seeds)
    lam = 1.0 if req.physics == "advection" else 1.0 * math.sqrt(2) + 1.2 + 0.2 * req.strength
    cfl = 0.1 if req.stepper == "rk4" else 1.0
    return cfl * h / ((2 * req.degree + 1) * lam)


def footprint(req: Request) -> int:
    """Device bytes a request holds while in flight."""
    nc = 4 if req.physics == "euler" else 1
    nb = (req.degree + 1) * (req.degree + 2) // 2
    bl = nb * nc
    n = req.n_seeds
    N = n * bl
    vqp = n * 6 * {1: 3, 2: 6, 3: 12}[req.degree]
    fqp = n * 6 * {1: 2, 2: 4, 3: 6}[req.degree]
    geo = vqp * 5 * 8 + fqp * 7 * 8 + n * 6 * 24 + n * nb * nb * 16
    fields = 12 * N * 8
    if req.stepper == "dirk3":
        nnzb = 7 * n
        # Jacobian, ILU(0) factors, the split form's E_i blocks, Krylov basis
        # and the sweep-form timing copy
        fields += 2 * nnzb * bl * bl * 8 + n * bl * bl * 8 + 33 * N * 8
    return int(1.15 * (geo + fields)) + (8 << 20)


def run_request(req: Request, device: int = 0) -> None:
    """Solve one request end to end on its own context and stream."""
    import torch
    stream = torch.cuda.Stream(device)
    with torch.cuda.stream(stream):
        ctx = cp.Context(device, stream)
        L = domain(req)
        seeds = cp.uniform_seeds(req.seed, req.n_seeds, L, L)
        mesh = cp.PolyMesh.voronoi(seeds, L, L, periodic=True)
        if req.physics == "advection":
            bx, by = math.cos(req.angle), math.sin(req.angle)
            eq = cp.ConstantAdvection(ctx, mesh, req.degree, bx, by)
            u = eq.interp(cp.INIT_GAUSSIAN, [100.0, 0.5, 0.5])
        else:
            vort = [req.strength, 5.0, 5.0, 1.0, 1.0, GAMMA, 10.0, 10.0]
            eq = cp.Euler(ctx, mesh, req.degree, dirichlet=(cp.INIT_VORTEX, vort), exact_jacobian=True)
            u = eq.interp(cp.INIT_VORTEX, vort)
        if req.stepper == "rk4":
            st = cp.RK4(eq)
        else:
            # the L-stable 3-stage SDIRK: the reference's 3-stage tableau has
            # |R(iy)| up to 1.78 on the imaginary axis, near which upwind DG
            # advection eigenvalues lie
            st = cp.DIRK(3, eq, l_stable=True, pc=cp.PC_ILU0, gmres_m=30, gmres_tol=1e-10)
        t = 0.0
        for _ in range(req.steps):
            st.advance(u, req.dt, t)
            req.newton += st.stats.newton_iterations
            req.gmres += st.stats.gmres_iterations
            t += req.dt
        stream.synchronize()
        req.result = u.cpu().numpy().ravel()
        del st, eq, u, mesh
        ctx.close()


class Server:
    """Admission by HBM footprint and slot count; one worker per slot."""

    def __init__(self, slots: int = 8, hbm_budget: int | None = None, device: int = 0):
        import torch
        self.slots = slots
        self.device = device
        if hbm_budget is None:
            free, _ = torch.cuda.mem_get_info(device)
            hbm_budget = int(0.8 * free)
        self.budget = hbm_budget
        self.in_use = 0
        self.cv = threading.Condition()
        self.active = 0
        self.peak_active = 0
        self.peak_bytes = 0

    def serve(self, requests: list[Request], realtime: bool = True) -> dict:
        """Run the stream; arrivals follow req.arrival when realtime."""
        pending = sorted(requests, key=lambda r: r.arrival)
        t0 = time.perf_counter()
        threads = []

        def worker(req: Request, nbytes: int):
            try:
                run_request(req, self.device)
            except Exception as e:  # reported per request; the server keeps going
                req.error = f"{type(e).__name__}: {e}"
            finally:
                req.done = time.perf_counter() - t0
                with self.cv:
                    self.in_use -= nbytes
                    self.active -= 1
                    self.cv.notify_all()

        for req in pending:
            nbytes = footprint(req)
            if nbytes > self.budget:
                req.error = "request larger than the device budget"
                req.done = req.admitted = time.perf_counter() - t0
                continue
            if realtime:
                wait = req.arrival - (time.perf_counter() - t0)
                if wait > 0:
                    time.sleep(wait)
            with self.cv:
                while self.active >= self.slots or self.in_use + nbytes > self.budget:
                    self.cv.wait()
                self.in_use += nbytes
                self.active += 1
                self.peak_active = max(self.peak_active, self.active)
                self.peak_bytes = max(self.peak_bytes, self.in_use)
            req.admitted = time.perf_counter() - t0
            th = threading.Thread(target=worker, args=(req, nbytes), daemon=True)
            th.start()
            threads.append(th)
        for th in threads:
            th.join()
        makespan = time.perf_counter() - t0
        ok = [r for r in requests if r.error is None]
        lat = np.array([r.done - r.arrival for r in ok]) if ok else np.zeros(1)
        return {"solves": len(ok), "failed": len(requests) - len(ok), "makespan_s": makespan,
                "solves_per_s": len(ok) / makespan, "p50_ms": float(np.percentile(lat, 50) * 1e3),
                "p99_ms": float(np.percentile(lat, 99) * 1e3), "peak_in_flight": self.peak_active,
                "peak_bytes": self.peak_bytes}
