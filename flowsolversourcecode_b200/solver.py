"""Host mirror of the reference's SIMPLE-loop subroutines over the C ABI.

Method names follow the Fortran subroutines they replace so a driver reads
like MainProgram/MainProgram.for:257-348:

    s = Solver(mesh, case)
    for nIter in range(1, IterMax + 1):
        s.SolveMomentumX(); s.SolveMomentumY(); s.SolveMomentumZ()
        s.SolveContinuity()
        source = s.PrintConvergenceHistory()
        if source < case.max_residual: break

Variables are the reference's ``character*10`` names ('velx', 'vely', 'velz',
'pressc', 'press').  All state lives on the GPU; nothing here computes on
the CPU, and every call raises :class:`FsError` on a non-zero status.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .case import Case
from .mesh import PolyMesh

VARIABLE = {"velx": L.VAR_U, "vely": L.VAR_V, "velz": L.VAR_W, "pressc": L.VAR_PC, "press": L.VAR_P,
            "temp": L.VAR_TEMP}


class Solver:
    def __init__(self, mesh: PolyMesh, case: Case, device: int = 0):
        self.lib = L.load()
        self.mesh = mesh
        self.case = case
        self._cfg = case.struct(mesh)
        ms, self._keep = L.mesh_struct(mesh)
        h = C.c_void_p()
        rc = self.lib.fs_create(C.byref(ms), C.byref(self._cfg), device, C.byref(h))
        L.check(rc, None, "fs_create")
        self.ctx = h
        n, f, b, w = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        self.lib.fs_sizes(self.ctx, C.byref(n), C.byref(f), C.byref(b), C.byref(w))
        self.N, self.F, self.B, self.W = n.value, f.value, b.value, w.value
        self.nIter = 0
        self.residuals: dict | None = None

    # ------------------------------------------------------------ lifetime
    def close(self):
        if getattr(self, "ctx", None):
            self.lib.fs_destroy(self.ctx)
            self.ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _chk(self, rc, what):
        L.check(rc, self.ctx, what)

    # ------------------------------------------------------------ drivers
    def SolveMomentumX(self):
        self._chk(self.lib.fs_solve_momentum(self.ctx, 0), "SolveMomentumX")

    def SolveMomentumY(self):
        self._chk(self.lib.fs_solve_momentum(self.ctx, 1), "SolveMomentumY")

    def SolveMomentumZ(self):
        self._chk(self.lib.fs_solve_momentum(self.ctx, 2), "SolveMomentumZ")

    def SolveContinuity(self):
        self._chk(self.lib.fs_solve_continuity(self.ctx), "SolveContinuity")

    def SolveEnergy(self):
        """SolveEnergy, 'temperature' (SelectEnergyEquationToSolve.for:4)."""
        self._chk(self.lib.fs_solve_energy(self.ctx), "SolveEnergy")

    energy = SolveEnergy

    def assemble_momentum(self, comp: int):
        self._chk(self.lib.fs_assemble_momentum(self.ctx, comp), "assemble_momentum")

    def assemble_continuity(self):
        self._chk(self.lib.fs_assemble_continuity(self.ctx), "assemble_continuity")

    def correct_continuity(self):
        self._chk(self.lib.fs_correct_continuity(self.ctx), "correct_continuity")

    def initialize_mdot(self):
        """CalculateInitialmdot from the current velocity fields (after set())."""
        self._chk(self.lib.fs_initialize_mdot(self.ctx), "initialize_mdot")

    # ------------------------------------------------------------ unsteady runs
    def advance_time(self, dt_next: float | None = None):
        """Time-step prologue of the unsteady loop (MainProgram.for:184-245):
        scheme selection, Crank-Nicolson extrapolation, updateVariablesInTime,
        dt bookkeeping, time += dt; the outer-iteration count restarts."""
        dt_next = self.case.dt if dt_next is None else dt_next
        self._chk(self.lib.fs_advance_time(self.ctx, float(dt_next)), "advance_time")
        self.nIter = 0

    def adaptive_time_step(self, courant: float = 2.0, min_factor: float = 0.5, max_factor: float = 5.0) -> float:
        """AdaptiveTimeStep (CalculateAdaptiveTimeStep.for:4-200) of a laminar,
        isothermal case: the next dt from the current mass fluxes, clamped to
        [min_factor dt, max_factor dt]; defaults are the reference's
        GlobalCourantNumber, minimumdtChangeFactor and maximumdtChangeFactor
        (ProblemDescriptionRoutine.for:544-546).  Pass it to advance_time."""
        dt = C.c_double(0.)
        self._chk(self.lib.fs_adaptive_time_step(self.ctx, float(courant), float(min_factor),
                                                 float(max_factor), C.byref(dt)), "adaptive_time_step")
        return dt.value

    def time_state(self) -> dict:
        t = (C.c_double * 4)()
        n = C.c_int32(0)
        self._chk(self.lib.fs_get_time(self.ctx, t, C.byref(n)), "get_time")
        return {"time": t[0], "dt": t[1], "dt_old": t[2], "dt_oldold": t[3], "ndt": n.value}

    def set_time_state(self, time: float, dt: float, dt_old: float, dt_oldold: float, ndt: int):
        t = (C.c_double * 4)(time, dt, dt_old, dt_oldold)
        self._chk(self.lib.fs_set_time(self.ctx, t, int(ndt)), "set_time")

    def run_time_step(self, itermax: int, tol: float | None = None, dt_next: float | None = None) -> list[dict]:
        """One time step: advance_time, then outer iterations until the
        stop metric falls below tol (do nIter=1,IterMax, MainProgram.for:257-325)."""
        self.advance_time(dt_next)
        return self.run(itermax, tol)

    def set_iteration(self, n: int):
        self.nIter = n
        self._chk(self.lib.fs_set_iteration(self.ctx, n), "set_iteration")

    def PrintConvergenceHistory(self) -> float:
        """Residual block + stop metric `source` (PrintConvergenceToFileAndScreen.for:613-700)."""
        r = L.FsResiduals()
        self._chk(self.lib.fs_residuals_get(self.ctx, C.byref(r)), "residuals")
        self.residuals = r.as_dict()
        return r.source

    def simple_iteration(self) -> dict:
        """One outer iteration (MainProgram.for:257-325) as a single C call."""
        r = L.FsResiduals()
        self.nIter += 1
        self._chk(self.lib.fs_simple_iteration(self.ctx, C.byref(r)), "fs_simple_iteration")
        self.residuals = r.as_dict()
        return self.residuals

    def simple_iteration_host(self, state: dict) -> dict:
        """One outer iteration on host-owned state arrays (copied in and out)."""
        r = L.FsResiduals()
        self.nIter += 1
        a = [state[k] for k in ("u", "v", "w", "p", "mdot", "bu", "bv", "bw", "bp", "bmdot")]
        self._chk(self.lib.fs_simple_iteration_host(self.ctx, *[L.dptr(x) for x in a], C.byref(r)),
                  "fs_simple_iteration_host")
        self.residuals = r.as_dict()
        return self.residuals

    def run(self, itermax: int, tol: float | None = None, callback=None) -> list[dict]:
        """Outer loop with the reference's stop test (MainProgram.for:322-325)."""
        tol = self.case.max_residual if tol is None else tol
        hist = []
        for _ in range(itermax):
            r = self.simple_iteration()
            hist.append(r)
            if callback:
                callback(self.nIter, r)
            if r["source"] < tol:
                break
        return hist

    # ------------------------------------------------------------ leaf routines
    def Gradient(self, variable: str, method: int, n_iter: int):
        self._chk(self.lib.fs_gradient(self.ctx, VARIABLE[variable], method, n_iter), "Gradient")

    def gradient_host(self, variable: str, method: int, n_iter: int, phi: np.ndarray, bphi: np.ndarray):
        phi = np.ascontiguousarray(phi, np.float64)
        bphi = np.ascontiguousarray(bphi, np.float64)
        g = np.zeros(3 * self.N)
        bg = np.zeros(3 * self.B)
        self._chk(self.lib.fs_gradient_host(self.ctx, VARIABLE[variable], method, n_iter, L.dptr(phi),
                                            L.dptr(bphi), L.dptr(g), L.dptr(bg)), "fs_gradient_host")
        return g, bg

    def UnderRelaxEquation(self, urf: float):
        self._chk(self.lib.fs_under_relax(self.ctx, urf), "UnderRelaxEquation")

    def SolveEquation(self, variable: str, rrf: float, itmax: int, solver: str):
        self._chk(self.lib.fs_solve_equation(self.ctx, VARIABLE[variable], rrf, itmax, L.SOLVER[solver]),
                  "SolveEquation")

    def solve_system(self, ac, anb, bc, rrf=0.1, itmax=100, solver="bicgs"):
        ac = np.ascontiguousarray(ac, np.float64)
        anb = np.ascontiguousarray(anb, np.float64)
        bc = np.ascontiguousarray(bc, np.float64)
        x = np.zeros(self.N)
        it = C.c_int()
        self._chk(self.lib.fs_solve_system_host(self.ctx, L.dptr(ac), L.dptr(anb), L.dptr(bc), L.dptr(x), rrf,
                                                itmax, L.SOLVER[solver], C.byref(it)), "fs_solve_system_host")
        return x, it.value

    # ------------------------------------------------------------ state
    def _size(self, name: str) -> int:
        N, F, B, W = self.N, self.F, self.B, self.W
        sizes = {"mdot": F, "gfactor": F, "gdiff": F, "sf": 3 * F, "ft": 3 * F, "anb": W * N,
                 "bu": B, "bv": B, "bw": B, "bp": B, "bpc": B, "bmdot": B, "bsf": 3 * B, "xc": 3 * N,
                 "btke": B, "bted": B, "bmut": B, "utau": B, "yplus": B,
                 "old": 7 * N, "oldold": 7 * N, "bold": 7 * B, "btemp": B}
        if name.endswith("grad"):
            return 3 * N
        return sizes.get(name, N)

    def get(self, name: str) -> np.ndarray:
        a = np.zeros(self._size(name))
        self._chk(self.lib.fs_get_field(self.ctx, L.FIELD_ID[name], L.dptr(a), a.shape[0]), f"get {name}")
        return a

    def set(self, name: str, arr) -> None:
        a = np.ascontiguousarray(arr, np.float64)
        self._chk(self.lib.fs_set_field(self.ctx, L.FIELD_ID[name], L.dptr(a), a.shape[0]), f"set {name}")

    # fields that carry information from one outer iteration to the next
    RESTART_FIELDS = ("u", "v", "w", "p", "mdot", "bu", "bv", "bw", "bp", "bmdot", "kx")
    RESTART_TURB = ("tke", "ted", "mut", "btke", "bted", "bmut", "utau", "yplus")
    RESTART_ENERGY = ("temp", "btemp")
    # unsteady runs: the old time levels (ReadSolutionToContinue.for:59-108)
    RESTART_UNSTEADY = ("old", "oldold", "bold")

    def write_solution(self, path: str) -> None:
        """writeSolution (WriteAndReadSolution/WriteSolutionToContinue.for:4):
        every array an outer iteration reads from the previous one -- the
        cell, face and boundary fields, BICGSTAB_OMP's persistent vector, the
        k-epsilon fields and wall-function state -- and the iteration count,
        to a .npz file.  Gradients, D, u* and the matrices are rebuilt by the
        next iteration before they are read, so they are not stored."""
        names = self.RESTART_FIELDS + (self.RESTART_TURB if self.case.turbulence else ())
        names += self.RESTART_ENERGY if self.case.energy else ()
        names += self.RESTART_UNSTEADY if self.case.unsteady else ()
        data = {k: self.get(k) for k in names}
        data["nIter"] = np.array([self.nIter], np.int64)
        if self.case.unsteady:
            t = self.time_state()
            data["time"] = np.array([t["time"], t["dt"], t["dt_old"], t["dt_oldold"]])
            data["ndt"] = np.array([t["ndt"]], np.int64)
        np.savez(path, **data)

    def read_solution(self, path: str) -> None:
        """readSolution: restore a state written by write_solution, so the
        next outer iterations repeat those of the run that wrote it."""
        with np.load(path) as f:
            for k in f.files:
                if k not in ("nIter", "time", "ndt"):
                    self.set(k, f[k])
            self.set_iteration(int(f["nIter"][0]))
            if "time" in f.files:
                self.set_time_state(*[float(x) for x in f["time"]], int(f["ndt"][0]))

    def state(self) -> dict:
        return {k: self.get(k) for k in ("u", "v", "w", "p", "mdot", "bu", "bv", "bw", "bp", "bmdot")}

    def connectivity(self) -> dict:
        N, W, F = self.N, self.W, self.F
        out = {"ncf": np.zeros(N, np.int32), "cf": np.zeros(N * W, np.int32), "cn": np.zeros(N * W, np.int32),
               "own_slot": np.zeros(F, np.int32), "nbr_slot": np.zeros(F, np.int32)}
        self._chk(self.lib.fs_get_connectivity(self.ctx, *[L.iptr(out[k]) for k in
                                                           ("ncf", "cf", "cn", "own_slot", "nbr_slot")]),
                  "connectivity")
        return out

    def mg_info(self) -> dict:
        """Multigrid hierarchy shapes: level sizes and ELL widths, and the
        coarsest level of the AMG preconditioner (dense inverse when direct)."""
        n = C.c_int()
        sizes = np.zeros(16, np.int32)
        widths = np.zeros(16, np.int32)
        lc, direct = C.c_int(), C.c_int()
        self._chk(self.lib.fs_mg_levels(self.ctx, C.byref(n), L.iptr(sizes), 16), "mg_levels")
        self._chk(self.lib.fs_mg_info(self.ctx, L.iptr(widths), 16, C.byref(lc), C.byref(direct)), "mg_info")
        k = n.value
        return {"sizes": sizes[:k].tolist(), "widths": widths[:k].tolist(), "prec_coarsest": lc.value,
                "direct": bool(direct.value)}

    def mg_coarse_matrix(self, level: int) -> dict:
        """AssembleAgglomeratedLHS of the last assembled system: the matrix of
        multigrid level `level` >= 1 (ac, n_nbr, nbr and anb slot-major)."""
        info = self.mg_info()
        sizes = np.zeros(16, np.int32)
        nl = C.c_int()
        self._chk(self.lib.fs_mg_levels(self.ctx, C.byref(nl), L.iptr(sizes), 16), "mg_levels")
        n, w = int(sizes[level]), int(info["widths"][level])
        out = {"ac": np.zeros(n), "n_nbr": np.zeros(n, np.int32), "nbr": np.zeros(n * w, np.int32),
               "anb": np.zeros(n * w)}
        self._chk(self.lib.fs_mg_coarse_matrix(self.ctx, level, L.dptr(out["ac"]), L.iptr(out["n_nbr"]),
                                               L.iptr(out["nbr"]), L.dptr(out["anb"]), n, w), "mg_coarse_matrix")
        return out

    def set_launch_shape(self, shape: int):
        """Threads per SM of the persistent cooperative solver kernels in units
        of 256 (1..4; 0: the default 1024), one CTA per SM."""
        self._chk(self.lib.fs_set_launch_shape(self.ctx, shape), "fs_set_launch_shape")

    def set_pc_history(self, m: int):
        """Start each AMG-BiCGSTAB p' solve from the least-squares combination of
        the m (0..7) previous p' solutions (and the learned guess when on)."""
        self._chk(self.lib.fs_set_pc_history(self.ctx, int(m)), "fs_set_pc_history")

    # ------------------------------------------------------------ learned p' guess
    def nn_create(self, snapshot_capacity: int = 0, seed: int = 0):
        """Network for the learned p' initial guess, with room for
        `snapshot_capacity` training snapshots of this mesh."""
        self._chk(self.lib.fs_nn_create(self.ctx, snapshot_capacity, seed), "fs_nn_create")

    def nn_mode(self, capture: bool = False, use: bool = False):
        self._chk(self.lib.fs_nn_mode(self.ctx, int(capture), int(use)), "fs_nn_mode")

    def nn_snapshots(self) -> int:
        n = C.c_int32()
        self._chk(self.lib.fs_nn_snapshots(self.ctx, C.byref(n)), "fs_nn_snapshots")
        return n.value

    def nn_train(self, epochs: int, lr: float = 1e-3, seed: int = 0) -> tuple[float, float]:
        a, b = C.c_float(), C.c_float()
        self._chk(self.lib.fs_nn_train(self.ctx, epochs, lr, seed, C.byref(a), C.byref(b)), "fs_nn_train")
        return a.value, b.value

    def nn_params(self, set: np.ndarray | None = None) -> np.ndarray:
        out = np.zeros(L.FS_NN_NPARAM, np.float32)
        s = None if set is None else np.ascontiguousarray(set, np.float32)
        self._chk(self.lib.fs_nn_params(self.ctx, L.fptr(out), L.fptr(s), L.FS_NN_NPARAM), "fs_nn_params")
        return out

    def nn_eval(self, X: np.ndarray, wgt: np.ndarray, target: np.ndarray | None = None) -> dict:
        """Forward (and with a target, loss and gradient) on host inputs."""
        X = np.ascontiguousarray(X, np.float32)
        wgt = np.ascontiguousarray(wgt, np.float32)
        t = None if target is None else np.ascontiguousarray(target, np.float32)
        loss = np.zeros(1, np.float32)
        grad = np.zeros(L.FS_NN_NPARAM, np.float32)
        y = np.zeros(self.N, np.float32)
        self._chk(self.lib.fs_nn_eval_host(self.ctx, L.fptr(X), L.fptr(wgt), L.fptr(t), L.fptr(loss),
                                           L.fptr(grad), L.fptr(y)), "fs_nn_eval_host")
        return {"y": y, "loss": float(loss[0]) if t is not None else None, "grad": grad if t is not None else None}

    def nn_stats(self) -> dict:
        """Guessed p' solves, guesses dropped by the residual guard, the
        policy's average iterations with the guess and from zero, and how
        often the guess was parked for not reducing iterations."""
        u, f = C.c_int32(), C.c_int32()
        g, z, p = C.c_double(), C.c_double(), C.c_int32()
        self._chk(self.lib.fs_nn_stats(self.ctx, C.byref(u), C.byref(f)), "fs_nn_stats")
        self._chk(self.lib.fs_nn_policy(self.ctx, C.byref(g), C.byref(z), C.byref(p)), "fs_nn_policy")
        return {"uses": u.value, "fallbacks": f.value, "avg_iters_guessed": g.value, "avg_iters_zero": z.value,
                "parked": p.value}

    def phase_times(self) -> list[float]:
        a = (C.c_float * 5)()
        self.lib.fs_phase_times(self.ctx, a)
        return list(a)

    def timer_start(self):
        self._chk(self.lib.fs_timer_start(self.ctx), "timer_start")

    def timer_stop(self) -> float:
        ms = C.c_float()
        self._chk(self.lib.fs_timer_stop(self.ctx, C.byref(ms)), "timer_stop")
        return ms.value

    def solver_stats(self, reset: bool = True) -> dict:
        """Per NF (u, v, w, p', -): solve milliseconds (set-up kernels
        included), linear iterations and calls since the last reset, and
        `kernel_ms`, the main cooperative solver kernel alone."""
        ms = (C.c_float * 5)()
        kms = (C.c_float * 5)()
        it = np.zeros(5, np.int32)
        calls = np.zeros(5, np.int32)
        self._chk(self.lib.fs_solver_kernel_ms(self.ctx, kms), "solver_kernel_ms")
        self._chk(self.lib.fs_solver_stats(self.ctx, ms, L.iptr(it), L.iptr(calls), int(reset)), "solver_stats")
        return {"ms": list(ms), "iters": it.tolist(), "calls": calls.tolist(), "kernel_ms": list(kms)}

    def launch_count(self) -> int:
        return int(self.lib.fs_launch_count(self.ctx))

    def sync(self):
        self._chk(self.lib.fs_sync(self.ctx), "sync")
