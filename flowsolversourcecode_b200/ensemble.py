"""Batched ensemble of independent cavity cases on one GPU (no reference
counterpart: the reference solves one case per process).

    cases = build_cases(make_specs(64, seed=0))   # edges U{32..96}, lid U[0.5, 2], Re log-U[100, 2000]
    ens = Ensemble(cases, device=0)
    ens.autotune()                          # launch shape per case, by timing
    out = ens.run(iters=10, launches=5)     # one CUDA graph per 10 iterations of all cases

Every case keeps its own context (mesh, fields, matrices, multigrid hierarchy);
`fs_ensemble_run` captures `iters` SIMPLE iterations of all cases into one CUDA
graph and launches it `launches` times; `fs_ensemble_run_batched` (run(...,
batched=True)) does the same with the p' solves of all cases in one cooperative
launch, a group of CTAs per case.  Across GPUs the cases shard by size
(`shard`, longest processing time first) with no collective on the data path.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from concurrent.futures import ProcessPoolExecutor
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from . import case as cs
from .mesh import splitmix64


@dataclass
class CaseSpec:
    edge: int
    lid: float
    re: float

    @property
    def cells(self) -> int:
        return self.edge ** 3


def make_specs(n_cases: int = 64, seed: int = 0, edges=(32, 96), lid=(0.5, 2.0), re=(100.0, 2000.0)):
    """Seeded case parameters (three splitmix64 draws per case): edge uniform on
    the integers [edges], lid speed uniform on [lid], Reynolds number
    log-uniform on [re] (viscosity = lid/Re on the unit cube, rho = 1)."""
    z = splitmix64(seed, 3 * n_cases)
    u = (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)
    out = []
    for q in range(n_cases):
        a, b, c = u[3 * q], u[3 * q + 1], u[3 * q + 2]
        e = edges[0] + min(int(a * (edges[1] - edges[0] + 1)), edges[1] - edges[0])
        v = lid[0] + b * (lid[1] - lid[0])
        r = math.exp(math.log(re[0]) + c * (math.log(re[1]) - math.log(re[0])))
        out.append(CaseSpec(int(e), float(v), float(r)))
    return out


def shard(sizes, world: int) -> list[list[int]]:
    """Longest-processing-time partition of case indices over `world` ranks."""
    parts = [[] for _ in range(world)]
    load = [0] * world
    for q in sorted(range(len(sizes)), key=lambda i: (-sizes[i], i)):
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(q)
        load[r] += sizes[q]
    return [sorted(p) for p in parts]


def build_case(spec: CaseSpec, **kw):
    """Mesh and Case of one ensemble member: the 3-D cavity with SOU deferred
    correction from iteration 1, the FP32 AMG preconditioner, p' solves started
    from the least-squares combination of the 4 previous p' solutions, and the
    multi-RHS momentum solve unless overridden."""
    kw.setdefault("solver_cont", "amg32_bicgs")
    kw.setdefault("pc_history", 4)
    kw.setdefault("krylov_tol", 1e-8)
    kw.setdefault("krylov_maxit", 200)
    kw.setdefault("batched_momentum", True)
    kw.setdefault("conv_scheme", "sou")
    kw.setdefault("niter_start_hr", 1)
    return cs.cavity(spec.edge, re=spec.re, lid=spec.lid, **kw)


def _mesh_job(args):
    spec, kw = args
    return build_case(spec, **kw)


def build_cases(specs, workers: int | None = None, **kw):
    """Meshes in a process pool (spawned: safe before or after CUDA use)."""
    workers = workers or min(8, os.cpu_count() or 1)
    if workers <= 1 or len(specs) == 1:
        return [build_case(s, **kw) for s in specs]
    import multiprocessing as mp
    with ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn")) as ex:
        return list(ex.map(_mesh_job, [(s, kw) for s in specs]))


class Ensemble:
    def __init__(self, cases, device: int = 0):
        from .solver import Solver
        self.solvers = [Solver(m, c, device=device) for m, c in cases]
        self.lib = self.solvers[0].lib
        self.cells = [s.N for s in self.solvers]
        self.shapes = [0] * len(self.solvers)
        self.split = 1.0
        self.split_ms = {}

    def autotune(self, shapes=(1, 2, 3, 4), iters: int = 2) -> list[int]:
        """Pick each case's cooperative launch shape (256 x shape threads on
        every SM) by timing `iters` SIMPLE iterations per candidate (after one
        untimed iteration at that shape)."""
        best = []
        for s in self.solvers:
            t = {}
            for k in shapes:
                s.set_launch_shape(k)
                s.simple_iteration()
                s.timer_start()
                for _ in range(iters):
                    s.simple_iteration()
                t[k] = s.timer_stop()
            k = min(t, key=lambda q: (t[q], q))
            s.set_launch_shape(k)
            best.append(k)
        self.shapes = best
        return best

    def autotune_split(self, exponents=(0.75, 1.0, 1.25, 1.5), iters: int = 2) -> float:
        """Pick the exponent of the CTA split of the batched form (groups in
        proportion to cells^e) by timing one launch of an `iters`-iteration
        graph per candidate; the fastest is kept."""
        t = {}
        for e in exponents:
            L.check(self.lib.fs_ensemble_split(self.solvers[0].ctx, float(e)), self.solvers[0].ctx,
                    "fs_ensemble_split")
            t[e] = self.run(iters=iters, launches=1, batched=True)["ms"]
        best = min(t, key=lambda e: (t[e], -e))
        L.check(self.lib.fs_ensemble_split(self.solvers[0].ctx, float(best)), self.solvers[0].ctx,
                "fs_ensemble_split")
        self.split = best
        self.split_ms = t
        return best

    def run(self, iters: int, launches: int = 1, batched: bool = False) -> dict:
        """`iters` SIMPLE iterations of every case per graph launch.  batched:
        the p' solves of all cases run as one cooperative launch with a CTA
        group per case (`fs_ensemble_run_batched`); otherwise the cases run
        one after another (`fs_ensemble_run`)."""
        n = len(self.solvers)
        T = iters * launches
        arr = (C.c_void_p * n)(*[s.ctx.value for s in self.solvers])
        src = np.zeros(n * T)
        pci = np.zeros(n * T, np.int32)
        ms = C.c_float()
        fn = "fs_ensemble_run_batched" if batched else "fs_ensemble_run"
        rc = getattr(self.lib, fn)(arr, n, iters, launches, L.dptr(src), L.iptr(pci), C.byref(ms))
        L.check(rc, self.solvers[0].ctx, fn)
        return {"source": src.reshape(n, T), "pc_iters": pci.reshape(n, T), "ms": ms.value,
                "cell_iters_per_s": sum(self.cells) * T / (ms.value * 1e-3)}

    def close(self):
        for s in self.solvers:
            s.close()
        self.solvers = []
