"""Benchmark: SIMPLE outer iterations per second on the 128^3 lid-driven cavity.

A step is one SIMPLE outer iteration (MainProgram.for:257-325: X/Y/Z momentum
assembly and solves, Rhie-Chow + p' assembly, p' solve, corrections,
residuals) on the 2,097,152-cell cavity (Re=1000, SOU deferred correction,
SIMPLEC, urf 0.7/0.7).  Synthetic mesh, generated here.

Forms (same case, same initial state):
  fp64   the plain FP64 GPU path: momentum by multicolour SOR, p' by FP64
         BiCGSTAB right-preconditioned with one element-agglomeration AMG
         V-cycle (coarsest level inverted densely), tolerance 1e-8.  `value`.
  mixed  the chosen forms: FP32 V-cycle (FP32 coarse matrices) inside the
         FP64 BiCGSTAB, the three momentum components as one multi-RHS solve.
         Reported under "mixed" with its field error against fp64.
  mixed_rrf  the mixed form with the p' solve stopped at a relative residual
         of 1e-3 (the reference's default rrFContinuity) instead of 1e-8: an
         inexact inner solve inside the SIMPLE loop.  Reported under
         "mixed_rrf"; the time-to-residual leg shows whether the outer
         iteration count and the converged fields change.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                  [--ttr MAXIT] (default 6000; 0 skips the time-to-residual legs)
  python bench.py --ensemble 64 [--gpus N]     the batched-ensemble configuration
  python bench.py --case distorted             the same cavity on the jittered mesh
  python bench.py --case bfs                   the k-epsilon backward-facing step (512x96x48)
  python bench.py --learned [--case bfs] [--n N]   train the learned p' guess on snapshots, then the
                                               case with and without it (cavity: the mixed form at 1e-3)

b200 arm: `value` is device-timed (CUDA events on the solver's stream) with
the state resident in HBM; `e2e` runs the fp64 steps through the C ABI
fs_simple_iteration_host with the state in pinned host buffers, copies inside
the timed region.  On one GPU the time to residual 1e-6 follows, from the
initial state, for the fp64 form, fp64 with the p' solves started from the
least-squares combination of the 4 previous p' solutions (fp64_guess), fp64
with the p' solve to 1e-3 (fp64_rrf), the mixed form at 1e-3 (mixed_rrf) and
the same with the initial guess (mixed_rrf_guess), with each form's converged
fields against the fp64 form's (at 128^3 about 3,300 outer iterations per
form; `--ttr 0` skips it, `--ttr MAXIT` caps the iterations).  N>1
(torchrun) runs one independent replica per GPU (the single-mesh path does not
shard) and reports the aggregate over ranks with the max-over-ranks time.
reference arm: the CPU restatement of the reference's loop with the
reference's own p' solver (unpreconditioned BiCGSTAB, same 1e-8 tolerance;
the Fortran reference cannot be compiled: no Fortran compiler on the host),
its AxOMP loop on every host core as the reference's OpenMP build runs it,
timed on the host, rank 0 only, within a 240 s budget.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

HBM_FALLBACK_GBS = 6650.0

FORMS = {
    "fp64": dict(solver_mom="sor", solver_cont="amg_bicgs", krylov_tol=1e-8, krylov_maxit=200),
    "mixed": dict(solver_mom="sor", solver_cont="amg32_bicgs", krylov_tol=1e-8, krylov_maxit=200,
                  batched_momentum=True),
    "mixed_rrf": dict(solver_mom="sor", solver_cont="amg32_bicgs", krylov_tol=1e-3, krylov_maxit=200,
                      batched_momentum=True),
    # the fp64 form with the same inexact p' solve: separates the gain of the
    # tolerance from the gain of the FP32 preconditioner in time to residual
    "fp64_rrf": dict(solver_mom="sor", solver_cont="amg_bicgs", krylov_tol=1e-3, krylov_maxit=200),
    # the mixed form with multicolour Gauss-Seidel smoothing in the FP32 V-cycle
    # (the distorted-mesh configuration names this smoother)
    "mixed_gs": dict(solver_mom="sor", solver_cont="amg32gs_bicgs", krylov_tol=1e-8, krylov_maxit=200,
                     batched_momentum=True),
    # the mixed form at 1e-3 whose p' solves start from the least-squares
    # combination of the 4 previous p' solutions (the learned network's guess
    # joins that basis when it is trained and on); the preconditioner's coarse
    # levels are rebuilt every 4th p' solve
    "mixed_rrf_guess": dict(solver_mom="sor", solver_cont="amg32_bicgs", krylov_tol=1e-3, krylov_maxit=200,
                            batched_momentum=True, pc_history=4, pc_refresh=4),
    # the plain FP64 form with the same initial guess (p' still to 1e-8)
    "fp64_guess": dict(solver_mom="sor", solver_cont="amg_bicgs", krylov_tol=1e-8, krylov_maxit=200, pc_history=4),
}
REFERENCE_SOLVERS = dict(solver_mom="sor", solver_cont="bicgs", krylov_tol=1e-8, krylov_maxit=300)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", HBM_FALLBACK_GBS)), "measured"
    return HBM_FALLBACK_GBS, "fallback"


def reduce_max(ms: float, dist=None, device="cpu") -> float:
    """Max of a per-rank device time over all ranks (the slowest replica sets
    the aggregate rate).  With no process group it is the local value."""
    if dist is None:
        return float(ms)
    import torch
    t = torch.tensor([ms], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def aggregate_rate(world: int, steps: int, ms_max: float) -> float:
    """Whole-job SIMPLE iterations per second: every rank runs `steps`
    iterations of its own replica; the job takes the slowest rank's time."""
    return world * steps / (ms_max * 1e-3)


def workload(n: int, form: str = "fp64", kind: str = "cubic", re_h: float = 5000.0):
    """The n^3 cavity (Re 1000, SOU); distorted: interior nodes jittered by
    U(-0.2h, 0.2h) from seed 0 (non-orthogonal correction is always on:
    MethodCalcGradient 2 and MethodDecomposeS 3); bfs: the backward-facing
    step 4n x 3n/4 x 3n/8 (512x96x48 at n=128), k-epsilon with wall functions,
    Re_H 5000, inlet u = 1 + 5% U(-1,1) from seed 0.  Returns (mesh, case,
    initial state or None)."""
    from flowsolversourcecode_b200 import case as cs
    kw = dict(REFERENCE_SOLVERS if form == "reference" else FORMS[form])
    if kind == "bfs":
        kw.pop("batched_momentum", None)      # k-epsilon runs the per-component momentum solves
        mesh, case = cs.bfs(4 * n, 3 * n // 4, 3 * n // 8, re_h=re_h, **kw)
        return mesh, case, cs.bfs_initial_state(mesh, case, seed=0)
    mesh, case = cs.cavity3d_distorted(n, seed=0, **kw) if kind == "distorted" else cs.cavity3d(n, **kw)
    return mesh, case, None


def workload_name(n: int, kind: str) -> str:
    if kind == "bfs":
        return (f"bfs_{4 * n}x{3 * n // 4}x{3 * n // 8} backward-facing step, channel 30H x 3H x 2H, k-epsilon "
                f"with equilibrium wall functions, Re_H=5000, inlet u=1+5% U(-1,1) seed 0")
    return (f"cavity3d_{n}" + ("_distorted (interior nodes jittered +-20% h, seed 0)" if kind == "distorted" else "")
            + " lid-driven cavity, Re=1000")


def start(obj, init):
    """Apply an initial state (set every field, then CalculateInitialmdot)."""
    if init:
        for k, v in init.items():
            obj.set(k, v)
        obj.initialize_mdot()
    return obj


class Clocks:
    """nvidia-smi sampler running during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self) -> dict:
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            c = [x.strip() for x in line.split(",")]
            if len(c) < 9:
                continue
            try:
                sm.append(float(c[1]))
                mx = float(c[2])
            except ValueError:
                continue
            for nm, v in zip(names, c[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- algorithmic bytes
def row_bytes(w: int, r: int) -> int:
    """One ELL row: diagonal (r bytes), w coefficients (r) and w int32 indices.
    The fixed-width row loops read all w slots (padded slots hold index -1)."""
    return r + (r + 4) * w


def vcycle_bytes(mg: dict, W: int, N: int, r: int) -> float:
    """Compulsory HBM bytes of one preconditioner V-cycle (PCycle, one pre- and
    one post-sweep): every array a phase touches is read or written once.
      level 0   x0 = w in/ac          : in 8 + ac r + x r
                residual              : row + in 8 + x r + r r
                prolong (own phase)   : x r (read) + x r (write) + parent 4
                sweep to `out` (FP64) : row + in 8 + x r + out 8
      level l   restrict into l       : per fine row r_{l-1} r + rlist 4;
                                        per row rptr 4 + b r + ac r + x r
                residual, prolong+sweep as level 0 with b r instead of in 8,
                                        the result into r (r bytes)
      coarsest  restrict as above; dense solve n_c^2 x 8 + b r + x r
    Gathers of neighbour values are L2 traffic and are not counted."""
    sizes, widths, lc = mg["sizes"], mg["widths"], mg["prec_coarsest"]
    total = 0.0
    for l in range(lc + 1):
        n, w = sizes[l], (W if l == 0 else widths[l])
        row = row_bytes(w, r)
        if l == 0:
            total += n * (8 + 2 * r)                                  # x0 = omega in / ac
            total += n * (row + 8 + 2 * r)                            # residual
            total += n * (2 * r + 4)                                  # prolong
            total += n * (row + 8 + r + 8)                            # sweep into out
            continue
        total += sizes[l - 1] * (r + 4) + n * (4 + 3 * r)            # restrict into l
        if l == lc and mg["direct"]:
            total += n * n * 8 + n * 2 * r
            continue
        total += n * (row + 3 * r)                                    # residual
        total += n * (2 * r + 4) + n * (row + 3 * r)                  # prolong + sweep
    return total


def amg_bicgstab_bytes(mg: dict, W: int, N: int, r: int, iters: int, calls: int) -> float:
    """k_amg_bicgstab: per BiCGSTAB iteration the Krylov algebra
      r0.r 16, p 32, v = A y (row + y 8 + v 8 + r0 8), s 24,
      t = A z (row + z 8 + t 8 + s 8), x/r update 56
    = 176 + 2 row bytes per row (FP64 matrix), plus two V-cycles; per launch
    the set-up (b, r, r0, p, v, x: 48) and dphi (8)."""
    row0 = row_bytes(W, 8)
    per_it = N * (176 + 2 * row0) + 2 * vcycle_bytes(mg, W, N, r)
    return per_it * iters + N * 56.0 * calls


def sor_bytes(W: int, N: int, sweeps: int, rhs: int = 1) -> float:
    """k_sor_colour (rhs=1) / k_sor3_colour (rhs=3) on the colour-major copy:
    a symmetric sweep visits every row twice (row + rhs x (bc 8 + x 8)), and
    the residual check once more (row + rhs x 16)."""
    row = row_bytes(W, 8) + (rhs - 1) * 8                # ac per component
    per_sweep = N * (2 * (row + rhs * 16) + row + rhs * 16)
    return per_sweep * sweeps


def solver_roofline(stats: dict, mg: dict | None, N: int, W: int, hbm: float, form: str,
                    ncu_traffic: dict | None):
    """Achieved HBM bandwidth of the solver kernel with the most device time
    (CUDA events around that kernel alone, on the solver stream)."""
    best = None
    for q in range(5):
        kms, its, calls = stats["kernel_ms"][q], stats["iters"][q], stats["calls"][q]
        if calls == 0 or kms <= 0:
            continue
        if q == 3:
            r = 4 if form == "mixed" else 8
            name = "k_amg_bicgstab<float>" if r == 4 else "k_amg_bicgstab<double>"
            nbytes = amg_bicgstab_bytes(mg, W, N, r, its, calls)
        elif form == "mixed" and q == 0:
            name, nbytes = "k_sor3_colour", sor_bytes(W, N, its, rhs=3)
        else:
            name, nbytes = "k_sor_colour", sor_bytes(W, N, its)
        if best is None or kms > best["ms"]:
            best = {"kernel": name, "ms": kms, "bytes": nbytes, "calls": calls, "iters": its}
    if best is None:
        return None
    achieved = best["bytes"] / (best["ms"] * 1e-3) / 1e9
    traffic = None
    if ncu_traffic and best["kernel"] in ncu_traffic:
        t = ncu_traffic[best["kernel"]]
        # DRAM bytes per (row x linear iteration) measured by ncu on a smaller
        # case of the same kernel, scaled to one launch here
        traffic = t["bytes_per_row_iter"] * N * best["iters"] / best["calls"]
    return {"bound": "hbm", "kernel": best["kernel"], "achieved": round(achieved, 1), "peak": hbm,
            "unit": "GB/s", "frac": round(achieved / hbm, 4), "traffic": traffic,
            "algorithmic_bytes_per_launch": best["bytes"] / best["calls"], "launches": best["calls"],
            "avg_launch_ms": best["ms"] / best["calls"],
            "iters_per_launch": best["iters"] / best["calls"]}


def host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_baseline_sample(n: int, kind: str = "cubic") -> dict:
    """The CPU restatement of the reference's loop on this host: the 2nd
    SIMPLE iteration of the same case (the 1st, from rest, is untimed) with
    the reference's OpenMP loop (AxOMP) on every host core, then the 3rd on
    one thread."""
    import oracle
    mesh, case, init = workload(n, "reference", kind)
    cores = host_cores()
    o = start(oracle.Oracle(mesh, case), init)
    o.simple_iteration()
    oracle.set_threads(cores)
    t0 = time.perf_counter()
    o.simple_iteration()
    dt = time.perf_counter() - t0
    oracle.set_threads(1)
    t0 = time.perf_counter()
    o.simple_iteration()
    dt1 = time.perf_counter() - t0
    o.close()
    return {"value": 1.0 / dt, "unit": "iter/s", "cores": cores, "kind": "port", "value_1thread": 1.0 / dt1,
            "sample": f"the 2nd SIMPLE outer iteration of the same {mesh.n_cells}-cell case on the CPU "
                      f"restatement (p' by the reference's unpreconditioned BiCGSTAB to 1e-8), its AxOMP loop "
                      f"on {cores} threads (all host cores); value_1thread: the 3rd iteration on 1 thread. "
                      f"Reference Fortran build unavailable (no Fortran compiler on the host)"}


def run_reference(args, rank: int) -> None:
    if rank != 0:
        return
    import oracle
    oracle.build()
    cores = host_cores()
    oracle.set_threads(cores)
    mesh, case, init = workload(args.n, "reference", args.case)
    o = start(oracle.Oracle(mesh, case), init)
    warm = max(args.warmup, 3)
    budget = 240.0           # seconds for warm-up and timed steps together
    t0 = time.perf_counter()
    w_run = 0
    for _ in range(warm):
        o.simple_iteration()
        w_run += 1
        if time.perf_counter() - t0 > budget / 4:
            break
    t_warm = time.perf_counter() - t0
    budget -= t_warm
    k_run = args.steps
    times = []
    for k in range(args.steps):
        t = time.perf_counter()
        o.simple_iteration()
        times.append(time.perf_counter() - t)
        if sum(times) > budget and k + 1 < args.steps:
            k_run = k + 1
            break
    total = sum(times)
    val = k_run / total
    line = {
        "impl": "reference", "metric": "SIMPLE iters/s", "value": val, "unit": "iter/s", "n_gpus": args.gpus,
        "steps": k_run, "warmup": w_run, "ms_per_step": 1e3 * total / k_run,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{workload_name(args.n, args.case)}, {mesh.n_cells} cells, SOU, SIMPLEC",
                   "cells": mesh.n_cells,
                   "solvers": "momentum sor, p' bicgs (the reference's unpreconditioned BiCGSTAB) to 1e-8",
                   "budget": f"{k_run} of {args.steps} requested timed steps and {w_run} of {warm} warm-up steps "
                             f"fit the 240 s budget of this arm"},
        "cpu_baseline": {"value": val, "unit": "iter/s", "cores": cores, "kind": "port",
                         "sample": f"{k_run} SIMPLE iterations after {w_run} untimed on the CPU restatement, its "
                                   f"AxOMP loop (the reference's OpenMP region) on {cores} threads, all host cores; "
                                   f"reference Fortran build unavailable (no Fortran compiler on the host)"},
        "e2e": {"value": val, "unit": "iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "warmup_s": t_warm,
    }
    print(json.dumps(line), flush=True)


def device_leg(s, steps: int, warm: int, barrier, local: int):
    """Warm up, then time `steps` SIMPLE iterations with CUDA events on the
    solver stream; clocks sampled during the timed region."""
    for _ in range(warm):
        s.simple_iteration()
    s.sync()
    s.solver_stats(reset=True)
    barrier()
    l0 = s.launch_count()
    ph = [0.0] * 5
    with Clocks(local) as clk:
        s.timer_start()
        last = None
        for _ in range(steps):
            last = s.simple_iteration()
            ph = [a + b for a, b in zip(ph, s.phase_times())]
        ms = s.timer_stop()
    return {"ms": ms, "launches": s.launch_count() - l0, "clocks": clk.summary(),
            "stats": s.solver_stats(reset=True), "phases": s.phase_times(), "phase_sum": ph, "last": last}


def assembly_roofline(leg: dict, N: int, F: int, steps: int, hbm: float) -> dict:
    """HBM fraction of everything in a SIMPLE iteration except the linear
    solves: gradients, momentum assembly with urf and D, Rhie-Chow + p'
    assembly, corrections and residuals.  Algorithmic bytes per iteration
    576 per interior face + 1432 per cell (each array read or written once per
    data-dependent phase, same-shape work sharing geometry); time = the
    momentum phase minus its solves, the continuity assembly phase, and the
    correction phase (CUDA events on the solver stream)."""
    ph, st = leg["phase_sum"], leg["stats"]
    ms = (ph[0] - sum(st["ms"][:3])) + ph[2] + ph[4]
    nbytes = (576.0 * F + 1432.0 * N) * steps
    achieved = nbytes / (ms * 1e-3) / 1e9
    return {"bound": "hbm", "achieved": round(achieved, 1), "peak": hbm, "unit": "GB/s",
            "frac": round(achieved / hbm, 4), "bytes_per_step": nbytes / steps, "ms_per_step": ms / steps}


def time_to_residual(Solver, mesh, case, local: int, maxit: int, tol: float = 1e-6, init=None,
                     keys=("u", "v", "w", "p")) -> tuple[dict, dict]:
    """Device time from the initial state until the stop metric drops below
    tol; returns the record and the fields reached."""
    s = start(Solver(mesh, case, device=local), init)
    s.timer_start()
    total, it, src = 0.0, 0, None
    for it in range(1, maxit + 1):
        r = s.simple_iteration()
        src = r["source"]
        if it % 200 == 0:
            total += s.timer_stop()
            s.timer_start()
        if src < tol:
            break
    total += s.timer_stop()
    fields = {k: s.get(k) for k in keys}
    s.close()
    return ({"seconds": total * 1e-3, "iterations": it, "reached": bool(src is not None and src < tol),
             "final_source": src}, fields)


def run_ensemble(args, world: int, rank: int, local: int, dist) -> None:
    """64 independent cavities of uneven size (edges U{32..96}, lid U[0.5, 2],
    Re log-uniform 100..2000, seed 0): FP64 outer iterations, FP32 AMG
    preconditioner, p' to `--ensemble-tol` (default 1e-3, the reference's
    rrFContinuity; the time-to-residual legs show the outer iterations and
    converged fields unchanged by it) from the least-squares combination of the
    4 previous p' solutions, multi-RHS momentum, launch shape autotuned per
    case, every `--steps` iterations of all of a GPU's cases one CUDA graph,
    timed in two forms -- cases in sequence, and the cases concurrently (the
    momentum solves of all cases in one cooperative launch and their p' solves
    in another, a CTA group per case, the remaining kernels as concurrent graph
    branches) -- and the faster one reported (both rates in `config`).
    Cases shard over ranks by size (longest processing time first); no
    collective on the data path.  Metric: cell-iterations per second, whole job."""
    import numpy as np
    from flowsolversourcecode_b200 import ensemble as E
    specs = E.make_specs(args.ensemble, seed=0)
    mine = E.shard([s.cells for s in specs], world)[rank]
    t0 = time.time()
    cases = E.build_cases([specs[q] for q in mine], krylov_tol=args.ensemble_tol)
    ens = E.Ensemble(cases, device=local)
    del cases
    t_setup = time.time() - t0
    shapes = ens.autotune(shapes=(1, 2, 3, 4), iters=1)
    split = ens.autotune_split(exponents=(0.75, 1.0, 1.25, 1.5), iters=2)
    launches = max(1, args.warmup)
    # both graph forms, each after one untimed launch of its own graph: cases in
    # sequence, and the p' solves of all cases in one launch (a CTA group each)
    timed = {}
    for batched in (False, True):
        ens.run(iters=args.steps, launches=1, batched=batched)
        if dist is not None:
            dist.barrier()
        with Clocks(local) as clk:
            out = ens.run(iters=args.steps, launches=launches, batched=batched)
        timed[batched] = (reduce_max(out["ms"], dist, f"cuda:{local}"), out, clk.summary())
    best = min(timed, key=lambda b: timed[b][0])
    ms, out, clocks = timed[best]
    cells = sum(ens.cells)
    total_cells = cells
    if dist is not None:
        import torch
        t = torch.tensor([float(cells)], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t)
        total_cells = t.item()
    T = args.steps * launches
    if rank == 0:
        line = {
            "metric": "ensemble cell-iterations/s", "value": total_cells * T / (ms * 1e-3), "unit": "cell-iter/s",
            "n_gpus": world, "steps": T, "warmup": args.steps, "ms_per_step": ms / T, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"ensemble of {len(specs)} lid-driven cavities, edges U{{32..96}}, lid U[0.5,2], "
                                   f"Re log-U[100,2000], seed 0",
                       "cases": len(specs), "cells_total": sum(s.cells for s in specs), "cases_rank0": len(mine),
                       "cells_rank0": cells, "graph": f"{args.steps} iterations of all rank cases per CUDA graph, "
                                                      f"{launches} launches",
                       "solvers": f"momentum multi-RHS SOR; p' FP64 BiCGSTAB + FP32 AMG V-cycle to "
                                  f"{args.ensemble_tol:g}, started from the least-squares combination of the 4 "
                                  f"previous p' solutions",
                       "launch_shapes_rank0": {str(k): shapes.count(k) for k in sorted(set(shapes))},
                       "cta_split_exponent_rank0": split,
                       "cta_split_ms_rank0": {str(k): round(v, 2) for k, v in ens.split_ms.items()},
                       "pc_launch": "the momentum solves of all cases in one cooperative launch and their p' "
                                    "solves in another, a CTA group per case; the other kernels of the cases as "
                                    "concurrent graph branches" if best else "the cases one after another",
                       "cell_iter_per_s_by_form": {
                           "sequential": total_cells * T / (timed[False][0] * 1e-3),
                           "batched_pc": total_cells * T / (timed[True][0] * 1e-3)},
                       "setup_s_rank0": round(t_setup, 1),
                       "source_rank0": {"min": float(np.min(out["source"][:, -1])),
                                        "max": float(np.max(out["source"][:, -1]))}},
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    ens.close()


def learned_workload(n: int, kind: str, re: float, form: str):
    """The case of the learned-guess leg: the step at Re_H = re (FP64 form), or
    the n^3 cavity (SOU from iteration 1) at Re = re in `form`."""
    from flowsolversourcecode_b200 import case as cs
    if kind == "bfs":
        return workload(n, "fp64", "bfs", re_h=re)
    mesh, case = cs.cavity(n, re=re, conv_scheme="sou", niter_start_hr=1, **FORMS[form])
    return mesh, case, None


def run_learned(args, local: int, n_re: int = 8, per_re: int = 50, epochs: int = 20) -> None:
    """The learned p' guess.  Step (`--case bfs`): snapshots from plain FP64
    runs at `n_re` Reynolds numbers Re_H ~ U[2000, 8000] (splitmix64 seed 1),
    evaluated at Re_H = 5000.  Cavity (`--case cubic`): snapshots from runs of
    the mixed form with the p' solve to 1e-3 and the history guess at Re
    log-uniform on [300, 3000] (seed 1), evaluated at Re = 1000 in the same
    form, whose p' initial guess is the least-squares combination of the 4
    previous p' solutions: the learned leg adds the network's guess to that
    basis, so the comparison shows what the network adds on top of it.  `per_re` snapshots per run (the p' solves of the first per_re+1
    SIMPLE iterations from the initial state); the network is trained on each
    run's snapshots in turn (parameters carried over); the evaluation case runs
    from the initial state with and without the guess, `--steps` iterations
    each after `--warmup`.  The guess only changes the p' starting vector: the
    solve still runs to the same tolerance."""
    import numpy as np
    from flowsolversourcecode_b200.mesh import uniform01
    from flowsolversourcecode_b200.solver import Solver
    kind = args.case
    if kind == "bfs":
        res, re_eval, form = [2000.0 + 6000.0 * float(x) for x in uniform01(1, n_re)], 5000.0, "fp64"
    else:
        n_re = 4
        res = [float(np.exp(np.log(300.0) + float(x) * (np.log(3000.0) - np.log(300.0)))) for x in uniform01(1, n_re)]
        re_eval, form = 1000.0, "mixed_rrf_guess"
    theta, train = None, []
    t0 = time.time()
    for q, re in enumerate(res):
        mesh, case, init = learned_workload(args.n, kind, re, form)
        s = start(Solver(mesh, case, device=local), init)
        s.nn_create(snapshot_capacity=per_re, seed=5)
        if theta is not None:
            s.nn_params(set=theta)
        s.nn_mode(capture=True, use=False)
        for _ in range(per_re + 1):
            s.simple_iteration()
        first, last = s.nn_train(epochs=epochs, lr=2e-3, seed=q)
        theta = s.nn_params()
        train.append({"re": round(re, 1), "snapshots": s.nn_snapshots(), "loss_first": first, "loss_last": last})
        s.close()
    t_train = time.time() - t0
    legs = {}
    for name, use in (("plain", False), ("learned", True)):
        mesh, case, init = learned_workload(args.n, kind, re_eval, form)
        s = start(Solver(mesh, case, device=local), init)
        if use:
            s.nn_create(0, seed=5)
            s.nn_params(set=theta)
            s.nn_mode(capture=False, use=True)
        for _ in range(max(args.warmup, 3)):
            s.simple_iteration()
        s.sync()
        s.solver_stats(reset=True)
        pits = 0
        with Clocks(local) as clk:
            s.timer_start()
            for _ in range(args.steps):
                pits += s.simple_iteration()["lin_iters"][3]
            ms = s.timer_stop()
        st = s.solver_stats(reset=True)
        legs[name] = {"value": args.steps / (ms * 1e-3), "ms_per_step": ms / args.steps, "pc_iters": pits,
                      "pc_ms_per_step": st["ms"][3] / args.steps, "clocks": clk.summary(),
                      "fields": {k: s.get(k) for k in ("u", "v", "w", "p")}}
        if use:
            legs[name]["policy"] = s.nn_stats()
        s.close()
    err = {k: float(np.linalg.norm(legs["learned"]["fields"][k] - legs["plain"]["fields"][k]) /
                    max(np.linalg.norm(legs["plain"]["fields"][k]), 1e-300)) for k in ("u", "v", "w", "p")}
    for v in legs.values():
        v.pop("fields")
    line = {
        "metric": "SIMPLE iters/s", "value": legs["learned"]["value"], "unit": "iter/s", "n_gpus": 1,
        "steps": args.steps, "warmup": max(args.warmup, 3), "ms_per_step": legs["learned"]["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": (workload_name(args.n, kind) if kind == "bfs" else
                                f"cavity3d_{args.n} lid-driven cavity, Re={re_eval:g}, SOU, the mixed form with the "
                                f"p' solve to 1e-3 and the history guess") + ", learned p' initial guess",
                   "form": form,
                   "training": {"re": [t["re"] for t in train], "snapshots_total": sum(t["snapshots"] for t in train),
                                "epochs_per_run": epochs, "runs": train, "seconds": round(t_train, 1)}},
        "plain": legs["plain"], "learned": legs["learned"],
        "learned_vs_plain_time": legs["learned"]["ms_per_step"] / legs["plain"]["ms_per_step"],
        "field_rel_l2_learned_vs_plain": err,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--case", default="cubic", choices=["cubic", "distorted", "bfs"])
    ap.add_argument("--ttr", type=int, default=6000, help="max iterations of the time-to-1e-6 legs (0: skip)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--learned", action="store_true",
                    help="train and measure the learned p' guess (--case bfs: FP64 step; cubic: the mixed form at 1e-3)")
    ap.add_argument("--ensemble", type=int, default=0, help="run the batched-ensemble configuration with this many cases")
    ap.add_argument("--ensemble-tol", type=float, default=1e-3,
                    help="p' tolerance of the ensemble cases (1e-3: the reference's default rrFContinuity)")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import numpy as np
    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)

    from flowsolversourcecode_b200 import build as fb
    fb.build()
    from flowsolversourcecode_b200.solver import Solver

    if args.ensemble > 0:
        run_ensemble(args, world, rank, local, dist)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        return

    def barrier():
        if dist is not None:
            dist.barrier()

    if args.learned:
        if args.case == "distorted" or world > 1:
            raise SystemExit("--learned runs with --case bfs or cubic on one GPU")
        run_learned(args, local)
        return

    warm = max(args.warmup, 3)
    kind = args.case
    mesh, case, init = workload(args.n, "fp64", kind)

    # ---------------- fp64 form: device-resident leg
    s = start(Solver(mesh, case, device=local), init)
    N, W, F = s.N, s.W, s.F
    mg = s.mg_info()
    d64 = device_leg(s, args.steps, warm, barrier, local)
    ms_max = reduce_max(d64["ms"], dist, f"cuda:{local}")
    fkeys = ("u", "v", "w", "p") + (("tke", "ted") if case.turbulence else ())
    fields64 = {k: s.get(k) for k in fkeys}

    # ---------------- fp64 form: end-to-end leg (host buffers through the C ABI)
    st = s.state()
    pinned = {}
    for k, v in st.items():
        pt = torch.empty(v.shape[0], dtype=torch.float64, pin_memory=True)
        a = pt.numpy()
        a[:] = v
        pinned[k] = (pt, a)
    host = {k: a for k, (_, a) in pinned.items()}
    for _ in range(2):
        s.simple_iteration_host(host)
    barrier()
    s.timer_start()
    for _ in range(args.steps):
        s.simple_iteration_host(host)
    e2e_ms = s.timer_stop()
    e2e_max = reduce_max(e2e_ms, dist, f"cuda:{local}")
    io_bytes = 8 * sum(a.shape[0] for a in host.values())
    s.close()

    # ---------------- mixed form: same case and initial state
    _, case_m, _ = workload(args.n, "mixed", kind)
    sm = start(Solver(mesh, case_m, device=local), init)
    dmx = device_leg(sm, args.steps, warm, barrier, local)
    msm_max = reduce_max(dmx["ms"], dist, f"cuda:{local}")
    err = {}
    for k, ref in fields64.items():
        x = sm.get(k)
        err[k] = float(np.linalg.norm(x - ref) / max(np.linalg.norm(ref), 1e-300))
    sm.close()

    # ---------------- mixed form with the inexact p' solve
    _, case_r, _ = workload(args.n, "mixed_rrf", kind)
    sr = start(Solver(mesh, case_r, device=local), init)
    drr = device_leg(sr, args.steps, warm, barrier, local)
    msr_max = reduce_max(drr["ms"], dist, f"cuda:{local}")
    err_r = {}
    for k, ref in fields64.items():
        x = sr.get(k)
        err_r[k] = float(np.linalg.norm(x - ref) / max(np.linalg.norm(ref), 1e-300))
    sr.close()

    # ---------------- mixed form with the Gauss-Seidel-smoothed FP32 V-cycle
    _, case_g, _ = workload(args.n, "mixed_gs", kind)
    sg = start(Solver(mesh, case_g, device=local), init)
    dgs = device_leg(sg, args.steps, warm, barrier, local)
    msg_max = reduce_max(dgs["ms"], dist, f"cuda:{local}")
    err_g = {}
    for k, ref in fields64.items():
        x = sg.get(k)
        err_g[k] = float(np.linalg.norm(x - ref) / max(np.linalg.norm(ref), 1e-300))
    sg.close()

    ttr = None
    if args.ttr > 0 and world == 1:
        # every form from the same initial state to the stop metric 1e-6; the
        # converged fields of each against the fp64 form's, and the times
        # against both fp64 legs (same p' tolerance 1e-8, and 1e-3)
        _, case_f, _ = workload(args.n, "fp64_rrf", kind)
        _, case_g, _ = workload(args.n, "mixed_rrf_guess", kind)
        _, case_fg, _ = workload(args.n, "fp64_guess", kind)
        ttr, tf = {}, {}
        legs = (("fp64", case), ("fp64_guess", case_fg), ("fp64_rrf", case_f), ("mixed_rrf", case_r),
                ("mixed_rrf_guess", case_g))
        for name, c in legs:
            ttr[name], tf[name] = time_to_residual(Solver, mesh, c, local, args.ttr, init=init, keys=fkeys)
        for name, _ in legs[1:]:
            ttr[name]["time_vs_fp64"] = ttr[name]["seconds"] / ttr["fp64"]["seconds"]
            ttr[name]["field_rel_l2_vs_fp64"] = {
                k: float(np.linalg.norm(tf[name][k] - tf["fp64"][k]) / max(np.linalg.norm(tf["fp64"][k]), 1e-300))
                for k in fkeys}
        for name in ("mixed_rrf", "mixed_rrf_guess"):
            ttr[name]["time_vs_fp64_rrf"] = ttr[name]["seconds"] / ttr["fp64_rrf"]["seconds"]
        ttr["mixed_rrf_guess"]["time_vs_fp64_guess"] = ttr["mixed_rrf_guess"]["seconds"] / ttr["fp64_guess"]["seconds"]
        ttr["forms"] = {"fp64": "the plain path (p' from zero to 1e-8)",
                        "fp64_guess": "fp64 with the p' solves started from the least-squares combination of the "
                                      "4 previous p' solutions",
                        "fp64_rrf": "fp64 with the p' solves to 1e-3 (the reference's default rrFContinuity)",
                        "mixed_rrf": "FP32 V-cycle + multi-RHS momentum, p' to 1e-3",
                        "mixed_rrf_guess": "mixed_rrf with the least-squares initial guess of fp64_guess, "
                                           "coarse preconditioner levels rebuilt every 4th p' solve"}
        ttr["tolerance"] = "stop metric (NstopType 4, normalised residual) below 1e-6 from the initial state"

    if rank == 0:
        hbm, src = peaks()
        ncu_t = None
        tp = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tp):
            with open(tp) as f:
                ncu_t = json.load(f)
        roof = solver_roofline(d64["stats"], mg, N, W, hbm, "fp64", ncu_t)
        roof_m = solver_roofline(dmx["stats"], mg, N, W, hbm, "mixed", ncu_t)
        for rf in (roof, roof_m):
            if rf:
                rf["peak_source"] = "measured (MEASURED_PEAKS.json hbm_gbs)" if src == "measured" else \
                    "fallback 6.65 TB/s"
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline_sample(args.n, kind)
        value = aggregate_rate(world, args.steps, ms_max)
        line = {
            "metric": "SIMPLE iters/s", "value": value, "unit": "iter/s", "n_gpus": world,
            "steps": args.steps, "warmup": warm, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"{workload_name(args.n, kind)}, {N} cells, {F} interior faces, "
                                   f"SOU deferred correction, SIMPLEC urf 0.7/0.7",
                       "cells": N, "faces": F,
                       "solvers": "momentum: multicolour SOR (rrF 0.01, 30 sweeps); p': FP64 BiCGSTAB "
                                  "right-preconditioned by one element-agglomeration AMG V-cycle, tol 1e-8"
                                  + ("; k, epsilon: multicolour SOR (rrF 0.1, 10 / 3 sweeps)" if case.turbulence else ""),
                       "mg_levels": mg["sizes"], "mg_prec_coarsest": mg["prec_coarsest"],
                       "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                       "l2": "inputs larger than L2 (working set ~2 GB)",
                       "lin_iters_last_step": d64["last"]["lin_iters"] if d64["last"] else None,
                       "turb_lin_iters_last_step": d64["last"]["turb_lin_iters"] if case.turbulence and d64["last"] else None,
                       "solver_ms_per_step": [round(x / args.steps, 3) for x in d64["stats"]["ms"]],
                       "phase_ms_last_step": [round(x, 3) for x in d64["phases"]]},
            "roofline": roof,
            "assembly_roofline": dict(assembly_roofline(d64, N, F, args.steps, hbm), **(
                {"note": "the timed correction phase also holds the k and epsilon equations (gradients, "
                         "assembly, SOR sweeps), which the byte count omits: a lower bound"}
                if case.turbulence else {})),
            "cpu_baseline": cpu,
            "e2e": {"value": aggregate_rate(world, args.steps, e2e_max), "unit": "iter/s",
                    "h2d_bytes_per_step": io_bytes, "d2h_bytes_per_step": io_bytes},
            "gpu_launches": d64["launches"],
            "clocks": d64["clocks"],
            "mixed": {"form": "FP32 AMG V-cycle (FP32 coarse matrices) inside FP64 BiCGSTAB to 1e-8"
                              + ("" if case.turbulence else "; multi-RHS momentum SOR"),
                      "value": aggregate_rate(world, args.steps, msm_max), "unit": "iter/s",
                      "ms_per_step": msm_max / args.steps,
                      "time_vs_fp64": msm_max / ms_max,
                      "field_rel_l2_vs_fp64": err,
                      "solver_ms_per_step": [round(x / args.steps, 3) for x in dmx["stats"]["ms"]],
                      "lin_iters_last_step": dmx["last"]["lin_iters"] if dmx["last"] else None,
                      "roofline": roof_m, "gpu_launches": dmx["launches"], "clocks": dmx["clocks"]},
            "mixed_rrf": {"form": "the mixed form with the p' solve to a relative residual of 1e-3 (the reference's "
                                  "default rrFContinuity) instead of 1e-8",
                          "value": aggregate_rate(world, args.steps, msr_max), "unit": "iter/s",
                          "ms_per_step": msr_max / args.steps, "time_vs_fp64": msr_max / ms_max,
                          "field_rel_l2_vs_fp64_same_steps": err_r,
                          "solver_ms_per_step": [round(x / args.steps, 3) for x in drr["stats"]["ms"]],
                          "lin_iters_last_step": drr["last"]["lin_iters"] if drr["last"] else None,
                          "gpu_launches": drr["launches"], "clocks": drr["clocks"]},
            "mixed_gs": {"form": "the mixed form with symmetric multicolour Gauss-Seidel smoothing on every level of "
                                 "the FP32 V-cycle (damped Jacobi in the mixed form)",
                         "value": aggregate_rate(world, args.steps, msg_max), "unit": "iter/s",
                         "ms_per_step": msg_max / args.steps, "time_vs_fp64": msg_max / ms_max,
                         "field_rel_l2_vs_fp64": err_g,
                         "solver_ms_per_step": [round(x / args.steps, 3) for x in dgs["stats"]["ms"]],
                         "lin_iters_last_step": dgs["last"]["lin_iters"] if dgs["last"] else None,
                         "gpu_launches": dgs["launches"], "clocks": dgs["clocks"]},
            "time_to_1e-6": ttr,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
