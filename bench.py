"""Benchmark: SIMPLE outer iterations per second on the 128^3 lid-driven cavity.

A step is one SIMPLE outer iteration (MainProgram.for:257-325: X/Y/Z momentum
assembly and solves, Rhie-Chow + p' assembly, p' solve, corrections,
residuals) on the 2,097,152-cell cavity (Re=1000, SOU deferred correction,
SIMPLEC, urf 0.7/0.7).  Synthetic mesh, generated here.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

b200 arm: `value` is device-timed (CUDA events on the solver's stream) with
the state resident in HBM; `e2e` runs the same steps through the C ABI
fs_simple_iteration_host with the state in pinned host buffers, copies inside
the timed region.  N>1 (torchrun) runs one independent replica per GPU (the
single-mesh path does not shard) and reports the aggregate over ranks with the
max-over-ranks time.  reference arm: the CPU restatement of the reference's
loop (the Fortran reference cannot be compiled in this image) timed on the
host, rank 0 only.
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


def workload(n: int):
    from flowsolversourcecode_b200 import case as cs
    mesh, case = cs.cavity3d(n, solver_mom="sor", solver_cont="bicgs")
    return mesh, case


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


def solver_roofline(stats: dict, N: int, W: int, hbm: float, ncu_traffic: dict | None):
    """Achieved HBM bandwidth of the solver kernel with the most device time.

    Algorithmic bytes per matrix row (FP64 values, int32 indices, W slots):
      matrix row          = 8 (ac) + 8W (anb) + 4W (cn) + 4 (ncf)
      BiCGSTAB iteration  = 2 SpMV x (row + 8 x_i + 8 y) + 8 (r0 in v.r0)
                            + 24 (s) + 48 (x, r) + 8 (r0) + 32 (p)
      BiCGSTAB set-up     = row + 8 (b) + 8 (x) + 24 (r0, r, p) + 8 (dphi)
      SOR sweep (fwd+bwd) = 2 x (row + 8 bc + 8 dphi + 4 colour list) + residual (row + 16)
    """
    row = 8 + 8 * W + 4 * W + 4
    per = {"bicgstab": 2 * (row + 16) + 8 + 24 + 48 + 8 + 32, "sor": 2 * (row + 20) + row + 16}
    best = None
    for q in range(5):
        ms, its, calls = stats["ms"][q], stats["iters"][q], stats["calls"][q]
        if calls == 0 or ms <= 0:
            continue
        kind = "bicgstab" if q == 3 else "sor"
        setup = (row + 48) if kind == "bicgstab" else 0
        nbytes = N * (per[kind] * its + setup * calls)
        if best is None or ms > best["ms"]:
            best = {"kernel": "k_bicgstab" if kind == "bicgstab" else "k_sor", "ms": ms, "bytes": nbytes,
                    "calls": calls, "iters": its}
    if best is None:
        return None
    achieved = best["bytes"] / (best["ms"] * 1e-3) / 1e9
    traffic = None
    if ncu_traffic and best["kernel"] in ncu_traffic:
        t = ncu_traffic[best["kernel"]]
        # measured bytes per row-iteration on a smaller case, scaled to these launches
        traffic = t["bytes_per_row_iter"] * N * best["iters"] / best["calls"]
    return {"bound": "hbm", "kernel": best["kernel"], "achieved": round(achieved, 1), "peak": hbm,
            "unit": "GB/s", "frac": round(achieved / hbm, 4),
            "traffic": traffic, "algorithmic_bytes_per_launch": best["bytes"] / best["calls"],
            "launches": best["calls"], "avg_launch_ms": best["ms"] / best["calls"]}


def cpu_baseline_sample(mesh, case) -> dict:
    import oracle
    o = oracle.Oracle(mesh, case)
    o.simple_iteration()                 # first iteration (CSR set-up), untimed
    t0 = time.perf_counter()
    o.simple_iteration()
    dt = time.perf_counter() - t0
    o.close()
    return {"value": 1.0 / dt, "unit": "iter/s", "cores": 1, "kind": "port",
            "sample": "1 SIMPLE outer iteration (the 2nd) of the same 128^3 case on the CPU restatement, 1 thread"}


def run_reference(args, rank: int) -> None:
    if rank != 0:
        return
    import oracle
    oracle.build()
    mesh, case = workload(args.n)
    o = oracle.Oracle(mesh, case)
    t0 = time.perf_counter()
    for _ in range(max(1, min(args.warmup, 1))):
        o.simple_iteration()
    t_warm = time.perf_counter() - t0
    budget = 150.0
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
        "steps": k_run, "warmup": max(1, min(args.warmup, 1)), "ms_per_step": 1e3 * total / k_run,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"cavity3d_{args.n} lid-driven cavity, {mesh.n_cells} cells, Re=1000, SOU, SIMPLEC",
                   "cells": mesh.n_cells, "solvers": "momentum sor, p' bicgs"},
        "cpu_baseline": {"value": val, "unit": "iter/s", "cores": 1, "kind": "port",
                         "sample": f"{k_run} of {args.steps} requested SIMPLE iterations (time budget {budget:.0f}s) "
                                   f"on the sequential CPU restatement; reference Fortran build unavailable "
                                   f"(no Fortran compiler in the image)"},
        "e2e": {"value": val, "unit": "iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "warmup_s": t_warm,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--no-cpu-baseline", action="store_true")
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

    mesh, case = workload(args.n)
    s = Solver(mesh, case, device=local)
    N, W = s.N, s.W
    warm = max(args.warmup, 3)

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---------------- device-resident leg
    for _ in range(warm):
        s.simple_iteration()
    s.sync()
    s.solver_stats(reset=True)
    barrier()
    l0 = s.launch_count()
    with Clocks(local) as clk:
        s.timer_start()
        last = None
        for _ in range(args.steps):
            last = s.simple_iteration()
        ms = s.timer_stop()
    launches = s.launch_count() - l0
    clocks = clk.summary()
    stats = s.solver_stats(reset=True)
    phases = s.phase_times()
    ms_max = reduce_max(ms, dist, f"cuda:{local}")

    # ---------------- end-to-end leg (host buffers through the C ABI)
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

    if rank == 0:
        hbm, src = peaks()
        ncu_t = None
        tp = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tp):
            with open(tp) as f:
                ncu_t = json.load(f)
        roof = solver_roofline(stats, N, W, hbm, ncu_t)
        if roof:
            roof["peak_source"] = f"{src} (MEASURED_PEAKS.json hbm_gbs)" if src == "measured" else "fallback 6.65 TB/s"
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline_sample(mesh, case)
        value = aggregate_rate(world, args.steps, ms_max)
        line = {
            "metric": "SIMPLE iters/s", "value": value, "unit": "iter/s", "n_gpus": world,
            "steps": args.steps, "warmup": warm, "ms_per_step": ms_max / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": f"cavity3d_{args.n} lid-driven cavity, {N} cells, {s.F} interior faces, "
                                   f"Re=1000, SOU deferred correction, SIMPLEC urf 0.7/0.7",
                       "cells": N, "faces": s.F, "solvers": "momentum sor (multicolour), p' bicgs",
                       "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                       "l2": "inputs larger than L2 (working set ~1.7 GB)",
                       "lin_iters_last_step": last["lin_iters"] if last else None,
                       "solver_ms_per_step": [round(x / args.steps, 3) for x in stats["ms"]],
                       "phase_ms_last_step": [round(x, 3) for x in phases]},
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": {"value": aggregate_rate(world, args.steps, e2e_max), "unit": "iter/s",
                    "h2d_bytes_per_step": io_bytes, "d2h_bytes_per_step": io_bytes},
            "gpu_launches": launches,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    s.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
