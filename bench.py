#!/usr/bin/env python
"""Benchmark: 3-stage DIRK steps/s of the 2D Euler isentropic vortex on
100,000 periodic Voronoi cells (p=3, 40x40 blocks), FP64, GMRES(30) + block
ILU(0), tolerance 1e-10, dt = 0.05 -- the reference's DG hot path end to end.

The 3-stage DIRK is Alexander's L-stable SDIRK3 by default.  The reference's
own 3-stage tableau (getDIRK, src/TimeIntegration.cpp:70-77) is not A-stable
(|R(-inf)| = 1.78): at this time step (CFL ~ 50 for the p=3 modes) its stiff
modes grow every step until the state turns non-physical; --tableau
reference selects it anyway.

Arms:
  default            this library on N GPUs (one process per GPU, replicas:
                     the path does not shard, every rank runs its own solve)
  --impl reference   the reference's CPU path, i.e. the oracle restatement
                     (oracle/), on this host's cores, on a bounded sample;
                     it builds its own meshes and never loads the library.

Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "DIRK3 steps/s Euler 100k-cell p3 mixed vs FP64 at 1e-8; batch solves/s, p99 ms"
WIDTH = 10.0
GAMMA = 1.4
VORTEX = [5.0, 5.0, 5.0, 1.0, 1.0, GAMMA, WIDTH, WIDTH]


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--cells", type=int, default=100000)
    ap.add_argument("--degree", type=int, default=3)
    ap.add_argument("--dt", type=float, default=0.05)
    ap.add_argument("--tableau", default="sdirk3", choices=["sdirk3", "reference"],
                    help="3-stage DIRK tableau: Alexander's L-stable SDIRK3 (default) or the reference's getDIRK(3), "
                         "which is not A-stable")
    ap.add_argument("--precision", default="f64", choices=["f64", "mixed", "pc32"],
                    help="f64; mixed = FP32 Jacobian and factors with FP64 FGMRES; pc32 = FP64 Jacobian with FP32 "
                         "factors (FP64 operator, FP32 preconditioner)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--systems", type=int, default=16, help="batch: independent systems per batched solve")
    ap.add_argument("--workload", default="dirk3", choices=["dirk3", "irk", "serve", "batch"],
                    help="dirk3: the 100k-cell vortex (default); irk: 2-stage Radau IIA, 500k cells, walls/inflow/"
                         "outflow, stage block-Jacobi GMRES(40) 1e-9; serve: Poisson stream of independent solves")
    ap.add_argument("--newton-tol", type=float, default=5e-13,
                    help="Newton tolerance on the residual's L2 norm (reference: 5e-13)")
    ap.add_argument("--reuse-jacobian", type=int, default=0,
                    help="rebuild the Jacobian and preconditioner every k-th Newton iteration (0 = every one)")
    ap.add_argument("--newton-rtol", type=float, default=None,
                    help="also stop Newton only once the last update is below this, relative to the stage vector "
                         "(default: 0, and 1e-8 for mixed, whose FP32-Jacobian Newton converges linearly)")
    ap.add_argument("--requests", type=int, default=512, help="serve: requests in the timed stream")
    ap.add_argument("--rate", type=float, default=200.0, help="serve: Poisson arrival rate, requests/s")
    ap.add_argument("--slots", type=int, default=8, help="serve: requests in flight at most")
    ap.add_argument("--max-seeds", type=int, default=50000, help="serve: largest mesh of the stream")
    ap.add_argument("--compare-fp64", type=int, default=0,
                    help="with --precision mixed: steps over which to measure the error against the FP64 path")
    a = ap.parse_args()
    if a.newton_rtol is None:
        # the FP32-Jacobian Newton converges linearly; 1e-8 on the update keeps
        # the 20-step result within 1e-8 of the FP64 path (5.2e-9 measured)
        a.newton_rtol = 1e-8 if a.precision == "mixed" else 0.0
    if a.workload == "irk":
        if a.cells == 100000:
            a.cells = 500000
        if a.degree == 3:
            a.degree = 2
        if a.dt == 0.05:
            # at 500k cells dt = 0.02 (CFL ~ 9) leaves block-Jacobi GMRES(40)
            # far from 1e-9 after 20,000 iterations; dt = 0.005 needs ~30
            a.dt = 0.005
    return a


def workload(a) -> dict:
    prec = {"mixed": "FP32 blocks + FGMRES", "pc32": "FP64 Jacobian + FP32 ILU factors"}.get(a.precision, "FP64")
    if a.workload == "batch":
        return {"workload": f"batched linear solves: {a.systems} independent SDIRK3 Newton systems of the p={a.degree} "
                            f"Euler vortex on periodic Voronoi meshes of 500-{a.max_seeds} cells (log-uniform, seeds "
                            f"100+k), each at the 100k case's dt/h; GMRES(30) + block ILU(0) tol 1e-10, {prec}; one "
                            f"step = all systems solved once",
                "systems": a.systems, "degree": a.degree, "max_seeds": a.max_seeds, "precision": a.precision,
                "l2": "small systems: the batch's matrices and factors (a few GB) stream once per iteration"}
    if a.workload == "serve":
        return {"workload": f"serving stream: {a.requests} independent solves, Poisson arrivals at {a.rate}/s; 50% "
                            f"advection (p in 1..3, random angle), 50% Euler vortex (p in 2..3, strength 1..5); "
                            f"Voronoi meshes of 500-{a.max_seeds} seeds (log-uniform); RK4 or DIRK3 (GMRES(30) + "
                            f"ILU(0) 1e-10), 10-100 steps; admission by HBM footprint, {a.slots} slots",
                "requests": a.requests, "rate": a.rate, "slots": a.slots, "max_seeds": a.max_seeds,
                "l2": "each request streams its own state; no L2 flush"}
    if a.workload == "irk":
        return {"workload": f"euler-density-bump Mach 0.3, [0,10]^2 slip walls / inflow / outflow, {a.cells} Voronoi "
                            f"cells (seed 5), p={a.degree}, 2-stage Radau IIA dt={a.dt}, GMRES(40) + block Jacobi on "
                            f"48x48 cell-coupled stage blocks tol 1e-9, Newton {a.newton_tol:g}, {prec}",
                "cells": a.cells, "degree": a.degree, "block": 4 * (a.degree + 1) * (a.degree + 2) // 2,
                "dt": a.dt, "gmres_m": 40, "gmres_tol": 1e-9, "preconditioner": "stage block Jacobi",
                "precision": a.precision, "jacobian": "exact", "newton_tol": a.newton_tol,
                "newton_rtol": a.newton_rtol, "reuse_jacobian": a.reuse_jacobian,
                "l2": "inputs larger than L2: each stage Jacobian streams ~16 GB per matvec"}
    tab = ("Alexander's L-stable SDIRK3 (gamma 0.435866521508459; the reference's getDIRK(3) tableau is not "
           "A-stable and diverges at this CFL)" if a.tableau == "sdirk3" else
           "the reference's getDIRK(3) tableau (order 2, not A-stable)")
    return {"workload": f"euler-isentropic-vortex periodic [0,10]^2, {a.cells} Voronoi cells (seed 2), p={a.degree}, "
                        f"3-stage DIRK = {tab}, dt={a.dt}, GMRES(30)+block ILU(0) tol 1e-10, Newton "
                        f"{a.newton_tol:g}, {prec}",
            "cells": a.cells, "degree": a.degree, "block": 4 * (a.degree + 1) * (a.degree + 2) // 2,
            "dt": a.dt, "tableau": a.tableau, "gmres_m": 30, "gmres_tol": 1e-10, "preconditioner": "ilu0",
            "precision": a.precision, "newton_tol": a.newton_tol, "newton_rtol": a.newton_rtol,
            "reuse_jacobian": a.reuse_jacobian,
            "jacobian": "exact (the reference's A_x entry and own-state neighbour blocks corrected; same residual "
                        "and converged solution, quadratic Newton); the CPU arm runs the same",
            "l2": "inputs larger than L2: the Jacobian and ILU factors stream ~9 GB each per sweep"}


# ------------------------------------------------------------------ clocks
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        sm.sort()
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": smax, "reasons": sorted(reasons),
                "samples": len(sm)}


def peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": d.get("hbm_gbs", 6650.0), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def profiled_traffic(name: str, key: str = "traffic_bytes_per_launch"):
    """dram bytes per launch (or per application) recorded from an ncu
    capture in profiles/"""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    for ln in open(p):
        if ln.startswith(key + ":"):
            try:
                return float(ln.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


# ------------------------------------------------------------------ CPU arm
def oracle_sample(a, n: int, threads: int, exact: bool = True):
    """Time the oracle (the reference's CPU algorithm, restated) on one step of
    the workload on an n-cell mesh at the workload's CFL: the time step is
    scaled by the cell size, dt_s = dt * sqrt(cells / n), so that dt/h -- and
    with it the Newton and GMRES iteration counts -- stay those of the full
    problem.  The oracle builds its own seeded Voronoi mesh; nothing of the
    library is loaded.  Returns (steps/s scaled to the full cell count, info)."""
    import oracle
    oracle.set_threads(threads)
    nthr = oracle.get_threads()
    dt = a.dt * (a.cells / n) ** 0.5
    if a.workload == "irk":
        inflow = [1.0, 0.3, 0.0, (1.0 / GAMMA) / (GAMMA - 1) + 0.5 * 0.3 ** 2]
        codes = [-2, -3, -2, -4]  # wall, outflow, wall, inflow (bottom, right, top, left)
        om = oracle.Mesh.voronoi(oracle.uniform_seeds(5, n, WIDTH, WIDTH), WIDTH, WIDTH, periodic=False,
                                 side_codes=codes)
        oe = oracle.Equation(om, 2, a.degree, gamma=GAMMA, dkind=0, dparams=inflow, inflow=inflow,
                             exact_jacobian=exact)
        u = oe.interp(3, [0.1, 0.5, 5.0, 5.0, 0.3, GAMMA])
        st = oracle.Stepper(oe, 6, pc=3, gmres_m=40, gmres_tol=1e-9, gmres_maxit=20000)
    else:
        om = oracle.Mesh.voronoi(oracle.uniform_seeds(2, n, WIDTH, WIDTH), WIDTH, WIDTH, periodic=True)
        oe = oracle.Equation(om, 2, a.degree, gamma=GAMMA, dkind=2, dparams=VORTEX, exact_jacobian=exact)
        u = oe.interp(2, VORTEX)
        st = oracle.Stepper(oe, 10 if a.tableau == "sdirk3" else 4, pc=2, gmres_m=30, gmres_tol=1e-10,
                            gmres_maxit=90000)
    t0 = time.perf_counter()
    u = st.advance(u, dt, 0.0)
    dt1 = time.perf_counter() - t0
    info = {"cells": n, "seconds": dt1, "dt": dt, "newton": int(st.stats[0]), "gmres": int(st.stats[1]),
            "converged": int(st.stats[3]), "threads": nthr}
    return 1.0 / (dt1 * a.cells / n), info


# sample sizes: one step of the all-core sample takes a few seconds on 16
# cores, the single-thread sample ~10 s
CPU_SAMPLE_CELLS = {"dirk3": 200, "irk": 400}
CPU_SAMPLE_CELLS_1T = {"dirk3": 100, "irk": 150}


def describe(info, a) -> str:
    return (f"one step of the same problem on a {info['cells']}-cell oracle mesh at the workload's CFL "
            f"(dt {info['dt']:.3f} = dt*sqrt({a.cells}/{info['cells']})), {info['seconds']:.1f} s on "
            f"{info['threads']} thread(s), Newton {info['newton']}, GMRES {info['gmres']}; scaled by "
            f"{a.cells}/{info['cells']} cells")


def cpu_baseline(a):
    """all-core and single-thread oracle samples for the GPU arm's line"""
    v, info = oracle_sample(a, CPU_SAMPLE_CELLS[a.workload], 0)
    v1, info1 = oracle_sample(a, CPU_SAMPLE_CELLS_1T[a.workload], 1)
    return {"value": v, "unit": "steps/s", "cores": info["threads"], "kind": "port", "sample": describe(info, a),
            "value_1thread": v1, "sample_1thread": describe(info1, a)}


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if a.workload in ("serve", "batch"):
        print(json.dumps({"impl": "reference", "unavailable": "the reference has no serving loop or batched "
                          "solver; its per-solve CPU cost is measured by the dirk3 and irk workloads"}), flush=True)
        return
    vals, info = [], None
    for k in range(a.warmup + a.steps):
        v, info = oracle_sample(a, CPU_SAMPLE_CELLS[a.workload], 0)
        if k >= a.warmup:
            vals.append(v)
    value = sum(vals) / len(vals)
    v1, info1 = oracle_sample(a, CPU_SAMPLE_CELLS_1T[a.workload], 1)
    # the reference's own (inexact) Euler Jacobian on the all-core sample:
    # same converged solution, linearly converging Newton
    vr, infor = oracle_sample(a, CPU_SAMPLE_CELLS[a.workload], 0, exact=False)
    out = {"metric": METRIC, "value": value, "unit": "steps/s", "impl": "reference", "n_gpus": a.gpus,
           "steps": a.steps, "warmup": a.warmup, "ms_per_step": 1000.0 / value, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Voronoi mesh)",
           "config": workload(a),
           "cpu_baseline": {"value": value, "unit": "steps/s", "cores": info["threads"], "kind": "port",
                            "sample": describe(info, a) + f"; mean of {a.steps} samples after {a.warmup}",
                            "value_1thread": v1, "sample_1thread": describe(info1, a),
                            "value_reference_jacobian": vr,
                            "sample_reference_jacobian": describe(infor, a) + " (the reference's inexact Euler "
                            f"Jacobian, Newton converged: {bool(infor['converged'])})"},
           "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


# ------------------------------------------------------------------ problems
def build_problem(a, cp, ctx):
    """(equation, stepper factory(mixed), initial state) of the workload."""
    if a.workload == "irk":
        # 2-stage Radau IIA on [0,10]^2: slip walls y=0,10, inflow x=0,
        # outflow x=10; uniform Mach 0.3 flow with a density bump
        inflow = [1.0, 0.3, 0.0, (1.0 / GAMMA) / (GAMMA - 1) + 0.5 * 0.3 ** 2]
        codes = [cp.BC_WALL, cp.BC_OUTFLOW, cp.BC_WALL, cp.BC_INFLOW]
        seeds = cp.uniform_seeds(5, a.cells, WIDTH, WIDTH)
        mesh = cp.PolyMesh.voronoi(seeds, WIDTH, WIDTH, periodic=False, side_codes=codes)
        eq = cp.Euler(ctx, mesh, a.degree, gamma=GAMMA, dirichlet=(cp.INIT_CONSTANT, inflow), inflow=inflow,
                      exact_jacobian=True)
        u0 = eq.interp(cp.INIT_DENSITY_BUMP, [0.1, 0.5, 5.0, 5.0, 0.3, GAMMA])

        def make(mixed):
            m32 = mixed == "mixed"
            return cp.IRK(2, eq, pc=cp.PC_STAGE_BJACOBI, precision=cp.F32 if m32 else cp.F64, gmres_m=40,
                          gmres_tol=1e-9, gmres_maxit=20000, flexible=m32, newton_tol=a.newton_tol,
                          reuse_jacobian=a.reuse_jacobian, newton_rtol=a.newton_rtol, pc_f32=mixed == "pc32")
        return eq, make, u0
    seeds = cp.uniform_seeds(2, a.cells, WIDTH, WIDTH)
    mesh = cp.PolyMesh.voronoi(seeds, WIDTH, WIDTH, periodic=True)
    eq = cp.Euler(ctx, mesh, a.degree, gamma=GAMMA, dirichlet=(cp.INIT_VORTEX, VORTEX), exact_jacobian=True)
    u0 = eq.interp(cp.INIT_VORTEX, VORTEX)

    def make(mixed):
        m32 = mixed == "mixed"
        return cp.DIRK(3, eq, l_stable=a.tableau == "sdirk3", pc=cp.PC_ILU0, precision=cp.F32 if m32 else cp.F64,
                       gmres_m=30, gmres_tol=1e-10, gmres_maxit=90000, flexible=m32, newton_tol=a.newton_tol,
                       reuse_jacobian=a.reuse_jacobian, newton_rtol=a.newton_rtol, pc_f32=mixed == "pc32")
    return eq, make, u0


# ------------------------------------------------------------------ GPU arm
def replica_throughput(local_ms: float, units: int, world: int, dist=None, device=None):
    """Replicas: every rank processes `units` on its own device; the job
    time is the slowest rank's device time.  Returns (max ms, units/s of the
    whole job)."""
    import torch
    if dist is not None and world > 1:
        dev = device if device is not None else ("cuda" if torch.cuda.is_available() else "cpu")
        t = torch.tensor([local_ms], dtype=torch.float64, device=dev)
        dist.barrier()
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        local_ms = float(t.item())
    return local_ms, world * units / (local_ms / 1000.0)


def run_serve(a):
    """Serving stream through cpolyg_b200.serve.Server: solves/s over the
    stream's makespan, p50/p99 latency from arrival to result on the host."""
    import torch

    from cpolyg_b200 import serve

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))
    # warm-up: a few small requests (library load, first-use kernel tuning)
    warm = serve.make_stream(max(a.warmup, 3), rate=1e6, seed=10_000 + rank, max_seeds=3000, max_steps=12)
    serve.Server(slots=a.slots, device=local).serve(warm, realtime=False)
    stream = serve.make_stream(a.requests, rate=a.rate, seed=rank, max_seeds=a.max_seeds)
    srv = serve.Server(slots=a.slots, device=local)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    stats = srv.serve(stream, realtime=True)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms_max, value = replica_throughput(stats["makespan_s"] * 1e3, stats["solves"], world, dist, f"cuda:{local}")
    if rank == 0:
        h2d = sum(r.n_seeds * 16 for r in stream)  # seeds go to the device as part of each request
        d2h = sum(r.result.nbytes for r in stream if r.result is not None)
        out = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": a.requests,
               "warmup": len(warm), "ms_per_step": ms_max / max(1, stats["solves"]), "higher_is_better": True,
               "scaling": "weak", "vs_baseline": None, "dtype": "f64",
               "data": "synthetic (seeded Voronoi meshes, analytic initial data, Poisson arrivals)",
               "config": dict(workload(a), parallelism=f"replicas x{world}"),
               "p50_ms": stats["p50_ms"], "p99_ms": stats["p99_ms"], "failed": stats["failed"],
               "peak_in_flight": stats["peak_in_flight"], "peak_bytes": stats["peak_bytes"],
               "newton_iterations": sum(r.newton for r in stream), "gmres_iterations": sum(r.gmres for r in stream),
               "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": h2d // max(1, a.requests),
                       "d2h_bytes_per_step": d2h // max(1, a.requests),
                       "note": "the serving loop is end to end: host seeds in, host coefficients out"},
               "clocks": clk}
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def _timed(fn, reps, stream):
    """device time per call of fn (CUDA events on the launching stream)"""
    import torch
    for _ in range(2):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps / 1000.0


def roofline(a, cp, ctx, eq, u, t, stream):
    """ILU(0) apply (two sync-free sweep launches) and BSR matvec of the
    step's Newton matrix B = M - gamma dt J at the current state, each
    against the measured HBM copy bandwidth.  Algorithmic bytes:
    sweeps nnzb*bl^2*s + 4*n*bl*8 (every factor block once; forward and
    backward read and write the vector), matvec nnzb*bl^2*s + 2*n*bl*8."""
    import torch
    if a.workload != "dirk3":
        return None
    mixed = a.precision == "mixed"
    s_a = 4 if mixed else 8
    s_p = 4 if a.precision in ("mixed", "pc32") else 8
    gamma = 0.435866521508459 if a.tableau == "sdirk3" else 0.717933260754229
    gmres_tol = 1e-10  # the stepper's
    J = eq.jacobian(u, t, scale=-a.dt * gamma, add_mass=True, precision=cp.F32 if mixed else cp.F64)
    P = cp.BlockILU0(J, precision=cp.F32 if s_p == 4 else cp.F64)
    x = torch.randn(u.numel(), dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    n, bl, nnzb = J.n_rows, J.bl, J.nb
    pk = peaks()
    reps = 20
    ctx.check(ctx._lib.cpg_ctx_set_deferred_checks(ctx.h, 1))  # no host read-back between the launches
    try:
        torch.cuda.nvtx.range_push("roofline_sweep")
        t_sw = _timed(lambda: ctx.check(ctx._lib.cpg_precond_apply(ctx.h, P.h, cp.C.c_void_p(x.data_ptr()))),
                      reps, stream)
        torch.cuda.nvtx.range_pop()
        ctx.sync()  # reads the sweeps' status word
        torch.cuda.nvtx.range_push("roofline_matvec")
        t_mv = _timed(lambda: ctx.check(ctx._lib.cpg_bsr_matvec(ctx.h, J.h, cp.C.c_void_p(x.data_ptr()),
                                                                cp.C.c_void_p(y.data_ptr()))), reps, stream)
        torch.cuda.nvtx.range_pop()
        # the GMRES step's operator P^{-1} A as the solve takes it at its
        # tolerance, and the split form whether or not it qualifies
        xp, yp = cp.C.c_void_p(x.data_ptr()), cp.C.c_void_p(y.data_ptr())
        torch.cuda.nvtx.range_push("roofline_operator")
        t_op = _timed(lambda: ctx.check(ctx._lib.cpg_precond_apply_op(ctx.h, P.h, J.h, xp, yp, gmres_tol)),
                      reps, stream)
        torch.cuda.nvtx.range_pop()
        t_split = None
        if P.split_ready(J):
            t_split = _timed(lambda: ctx.check(ctx._lib.cpg_precond_apply_op(ctx.h, P.h, J.h, xp, yp, 1.0)),
                             reps, stream)
        ctx.sync()
    finally:
        ctx.check(ctx._lib.cpg_ctx_set_deferred_checks(ctx.h, 0))
    form = int(ctx._lib.cpg_precond_sweep_form(P.h))
    cond = P.pivot_cond()
    split = P.split_ready(J) and 0.25 * 2.0 ** -52 * cond <= gmres_tol
    alg_sw = nnzb * bl * bl * s_p + 4 * n * bl * 8
    alg_mv = nnzb * bl * bl * s_a + 2 * n * bl * 8
    ach_sw, ach_mv = alg_sw / t_sw / 1e9, alg_mv / t_mv / 1e9
    # split rows: E_i and A's upper blocks ((nnzb - n) / 2, symmetric
    # pattern), x in, y out; the backward sweep also reads x once more
    alg_sr = (n + (nnzb - n) // 2) * bl * bl * s_a + 2 * n * bl * 8
    alg_op = (alg_sr + alg_sw + n * bl * 8) if split else (alg_mv + alg_sw)
    prec_sw = "FP32" if s_p == 4 else "FP64"
    kname = {1: "k_sweep (TMA ring)", 4: "k_sweep_direct", 5: "k_sweep_direct (2x rows)",
             6: "k_sweep_direct (4x rows)", 2: "k_rows per level", 3: "k_rows per level (wide)"}.get(form, "sweep")
    traffic = profiled_traffic(f"sweep_direct_{prec_sw.lower()}_bl{bl}_100k.md", "traffic_bytes_per_apply")
    roof = {"kernel": f"{kname}: ILU(0) apply, forward + backward sweep, {bl}x{bl} {prec_sw} factors "
                      f"(sweep form {form})",
            "bound": "hbm", "achieved": ach_sw, "peak": pk["hbm_gbs"], "unit": "GB/s",
            "frac": ach_sw / pk["hbm_gbs"], "peak_source": pk["source"], "algorithmic_bytes": alg_sw,
            "launch_ms": t_sw * 1e3, "launches_per_unit": 2 if form in (1, 4, 5, 6) else None,
            "traffic": traffic,
            "matvec": {"kernel": f"k_rows (BSR matvec, {bl}x{bl} {'FP32' if mixed else 'FP64'} blocks)",
                       "achieved": ach_mv, "frac": ach_mv / pk["hbm_gbs"], "algorithmic_bytes": alg_mv,
                       "launch_ms": t_mv * 1e3,
                       "traffic": profiled_traffic(f"bsr_matvec_{'f32' if mixed else 'f64'}_bl{bl}.md")},
            "operator": {"kernel": ("P^{-1} A, split form: k_rows_split (E + upper blocks of A), forward sweep, "
                                    "backward sweep adding x" if split else "P^{-1} A: BSR matvec, then ILU(0) apply"),
                         "split": split, "pivot_cond_max": cond, "gmres_tol": gmres_tol,
                         "launch_ms": t_op * 1e3, "algorithmic_bytes": alg_op,
                         "achieved": alg_op / t_op / 1e9, "frac": alg_op / t_op / 1e9 / pk["hbm_gbs"]}}
    if t_split is not None:
        # the split form timed even where its rounding (eps * cond) keeps the
        # solve on the plain product
        alg_spl = alg_sr + alg_sw + n * bl * 8
        t_sr = max(t_split - t_sw, 1e-9)
        roof["operator"]["split_form"] = {"used_by_the_solve": split, "launch_ms": t_split * 1e3,
                                          "algorithmic_bytes": alg_spl, "achieved": alg_spl / t_split / 1e9,
                                          "split_rows_ms": t_sr * 1e3,
                                          "split_rows_achieved": alg_sr / t_sr / 1e9}
    del P, J
    return roof


def run_batch(a):
    """Solves/s of a set of independent Newton systems of uneven size: one
    batched GMRES over the block-diagonal stack (segmented reductions, one
    host synchronisation per restart cycle) against the same systems solved
    one after another.  Inputs resident on the device; e2e copies the
    right-hand sides in and the solutions out."""
    import numpy as np
    import torch

    import cpolyg_b200 as cp

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    ctx = cp.Context(local)
    rng = np.random.default_rng(7)
    sizes = np.exp(rng.uniform(np.log(500), np.log(a.max_seeds), a.systems)).astype(int).tolist()
    prec = cp.F32 if a.precision == "mixed" else cp.F64
    flexible = a.precision == "mixed"
    Js = []
    for k, n in enumerate(sizes):
        m = cp.PolyMesh.voronoi(cp.uniform_seeds(100 + k, n, WIDTH, WIDTH), WIDTH, WIDTH, periodic=True)
        eq = cp.Euler(ctx, m, a.degree, gamma=GAMMA, dirichlet=(cp.INIT_VORTEX, VORTEX), exact_jacobian=True)
        u = eq.interp(cp.INIT_VORTEX, VORTEX)
        Js.append(eq.jacobian(u, 0.0, scale=-0.05 * (100000 / n) ** 0.5 * 0.435866521508459, add_mass=True,
                              precision=prec))
    Ps = [cp.BlockILU0(J, precision=prec) for J in Js]
    S = cp.BlockMatrix.stack(Js)
    PS = cp.BlockILU0(S, precision=prec)
    gen = torch.Generator("cuda").manual_seed(1)
    b = torch.randn(S.n_rows * S.bl, dtype=torch.float64, device="cuda", generator=gen)
    seg = S.seg_rows
    bl = S.bl
    stream = torch.cuda.current_stream()

    def one_by_one():
        its = 0
        for k, (J, P) in enumerate(zip(Js, Ps)):
            bk = b[seg[k] * bl:seg[k + 1] * bl]
            xk = torch.zeros_like(bk)
            its += J.gmres(bk, xk, 30, 1e-10, 90000, P, flexible=flexible)[0]
        return its

    def batched():
        x = torch.zeros_like(b)
        return sum(i for i, _ in S.gmres_batched(seg, b, x, 30, 1e-10, 90000, PS, flexible=flexible)), x

    for _ in range(a.warmup):
        one_by_one()
        batched()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = ctx.launches
    e0.record(stream)
    for _ in range(a.steps):
        its_b, _ = batched()
    e1.record(stream)
    torch.cuda.synchronize()
    ms_b = e0.elapsed_time(e1) / a.steps
    launches = ctx.launches - launches0
    e0.record(stream)
    for _ in range(a.steps):
        its_s = one_by_one()
    e1.record(stream)
    torch.cuda.synchronize()
    ms_s = e0.elapsed_time(e1) / a.steps
    clk = clocks.stop()
    # end to end: right-hand sides in from pinned host memory, solutions out
    bh = b.cpu().pin_memory()
    xh = torch.empty_like(bh).pin_memory()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(a.steps):
        bd = bh.cuda(non_blocking=True)
        x = torch.zeros_like(bd)
        S.gmres_batched(seg, bd, x, 30, 1e-10, 90000, PS, flexible=flexible)
        xh.copy_(x, non_blocking=True)
    torch.cuda.synchronize()
    e2e_s = (time.perf_counter() - t0) / a.steps
    ms_max, value = replica_throughput(ms_b, a.systems, world, dist)
    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": a.steps,
               "warmup": a.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None, "dtype": "f32 blocks, f64 vectors" if flexible else "f64",
               "data": "synthetic (seeded Voronoi meshes, analytic state)",
               "config": dict(workload(a), parallelism=f"replicas x{world}", sizes=sizes),
               "one_by_one": {"value": a.systems / (ms_s / 1e3), "unit": "solves/s", "ms_per_step": ms_s},
               "gmres_iterations": {"batched": its_b, "one_by_one": its_s},
               "e2e": {"value": a.systems / e2e_s, "unit": "solves/s", "h2d_bytes_per_step": int(bh.numel() * 8),
                       "d2h_bytes_per_step": int(xh.numel() * 8)},
               "gpu_launches": launches, "clocks": clk}
        print(json.dumps(out), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_ours(a):
    import numpy as np
    import torch

    import cpolyg_b200 as cp

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    ctx = cp.Context(local)
    mixed = a.precision == "mixed"  # FP32 Jacobian (matvec in FP32)
    eq, make_stepper, u0 = build_problem(a, cp, ctx)
    stepper = make_stepper(a.precision)
    u = u0.clone()
    stream = torch.cuda.current_stream()

    # mixed precision: error against the FP64 GPU path from the same state
    err_fp64 = None
    if a.precision != "f64" and a.compare_fp64 and rank == 0:
        ref_stepper = make_stepper("f64")
        ua, ub = u0.clone(), u0.clone()
        tt = 0.0
        for _ in range(a.compare_fp64):
            ref_stepper.advance(ua, a.dt, tt)
            stepper.advance(ub, a.dt, tt)
            tt += a.dt
        err_fp64 = float(torch.linalg.norm(ub - ua) / torch.linalg.norm(ua))
        del ref_stepper, ua, ub
        torch.cuda.empty_cache()

    t = 0.0
    for _ in range(a.warmup):
        stepper.advance(u, a.dt, t)
        t += a.dt
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = ClockSampler(local)
    clocks.start()
    time.sleep(0.3)
    launches0 = ctx.launches
    newton, gmres = [], []
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ev0.record(stream)
    for _ in range(a.steps):
        stepper.advance(u, a.dt, t)
        newton.append(stepper.stats.newton_iterations)
        gmres.append(stepper.stats.gmres_iterations)
        t += a.dt
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    launches = ctx.launches - launches0
    clk = clocks.stop()
    ms_max, value = replica_throughput(ms, a.steps, world, dist)

    # end to end through the C ABI with host buffers (cpg_step_host)
    e2e = None
    if not a.no_e2e:
        uh = torch.empty(u.numel(), dtype=torch.float64).pin_memory().numpy()
        uh[:] = u.cpu().numpy().ravel()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(a.steps):
            stepper.advance_host(uh, a.dt, t)
            t += a.dt
        torch.cuda.synchronize()
        e2e_s = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device="cuda")
        if dist:
            dist.all_reduce(e2e_s, op=dist.ReduceOp.MAX)
        e2e = {"value": world * a.steps / float(e2e_s.item()), "unit": "steps/s",
               "h2d_bytes_per_step": int(uh.nbytes), "d2h_bytes_per_step": int(uh.nbytes)}

    # roofline of the dominant kernel: the ILU(0) triangular sweeps (one
    # forward and one backward launch per application, ~40% of the step),
    # then the BSR matvec (~38%); both timed live with CUDA events on the
    # launching stream, on the step's own Newton matrix and its factors
    roof = None
    if rank == 0:
        roof = roofline(a, cp, ctx, eq, u, t, stream)

    if rank == 0:
        cpu = cpu_baseline(a) if (not a.no_cpu_baseline and world == 1) else None
        out = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": a.steps,
               "warmup": a.warmup, "ms_per_step": ms_max / a.steps, "higher_is_better": True, "scaling": "weak",
               "vs_baseline": None,
               "dtype": {"mixed": "f32 blocks, f64 vectors", "pc32": "f64 blocks, f32 factors, f64 vectors"}.get(
                   a.precision, "f64"),
               "data": "synthetic (seeded Voronoi mesh, analytic initial data)",
               "config": dict(workload(a), parallelism=f"replicas x{world}"),
               "newton_iterations_per_step": sum(newton) / a.steps, "gmres_iterations_per_step": sum(gmres) / a.steps,
               "newton_per_step": newton, "gmres_per_step": gmres,
               "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches, "clocks": clk}
        if err_fp64 is not None:
            out["error_vs_fp64"] = {"value": err_fp64, "steps": a.compare_fp64,
                                    "norm": "relative 2-norm of the coefficient vector"}
        print(json.dumps(out), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    a = parse()
    if a.impl == "reference":
        run_reference(a)
    elif a.workload == "serve":
        run_serve(a)
    elif a.workload == "batch":
        run_batch(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
