"""ctypes access to the CPU restatement of the reference SIMPLE loop.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference legs.  The product never imports it.
Parity is unpinned (see oracle.h): the reference is Fortran with no compiler
in this image and ships no golden vectors.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
_lib = None


def build() -> str:
    r = subprocess.run(["make", "-s", "-C", HERE], capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    return LIB


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = C.CDLL(LIB)
        lib.om_create.restype = C.c_void_p
        lib.om_create.argtypes = [C.c_void_p, C.c_void_p]
        lib.om_destroy.argtypes = [C.c_void_p]
        lib.om_array.restype = C.c_void_p
        lib.om_array.argtypes = [C.c_void_p, C.c_char_p, C.POINTER(C.c_long), C.POINTER(C.c_int)]
        lib.om_sizes.argtypes = [C.c_void_p] + [C.POINTER(C.c_int)] * 4
        for n in ("om_momentum", "om_assemble_momentum"):
            getattr(lib, n).argtypes = [C.c_void_p, C.c_int]
        for n in ("om_continuity", "om_assemble_continuity", "om_correct_continuity"):
            getattr(lib, n).argtypes = [C.c_void_p]
        lib.om_simple_iteration.restype = C.c_double
        lib.om_simple_iteration.argtypes = [C.c_void_p]
        lib.om_set_iter.argtypes = [C.c_void_p, C.c_int]
        lib.om_residuals.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        lib.om_lin_iters.argtypes = [C.c_void_p, C.c_int]
        lib.om_gradient.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int] + [C.c_void_p] * 4
        lib.om_solve_equation.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_double, C.c_int, C.c_int]
        lib.om_bicgstab.restype = C.c_int
        lib.om_bicgstab.argtypes = [C.c_void_p, C.c_int, C.c_double]
        lib.om_gmres.restype = C.c_int
        lib.om_gmres.argtypes = [C.c_void_p]
        lib.om_calc_residuals.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        lib.om_residuals_turb.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        lib.om_residuals_temp.argtypes = [C.c_void_p, C.POINTER(C.c_double)]
        lib.om_energy.argtypes = [C.c_void_p]
        lib.om_initialize_mdot.argtypes = [C.c_void_p]
        lib.om_turb_production.argtypes = [C.c_void_p]
        lib.om_neu_connectivity_literal.restype = C.c_int
        lib.om_neu_connectivity_literal.argtypes = [C.c_void_p] + [C.POINTER(C.c_int32)] * 8
        lib.om_advance_time.argtypes = [C.c_void_p, C.c_double]
        lib.om_adaptive_dt.restype = C.c_double
        lib.om_adaptive_dt.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_double]
        lib.om_get_time.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.POINTER(C.c_int)]
        lib.om_set_time.argtypes = [C.c_void_p, C.POINTER(C.c_double), C.c_int]
        lib.om_mg_setup.restype = C.c_int
        lib.om_mg_setup.argtypes = [C.c_void_p]
        lib.om_mg_level_size.restype = C.c_int
        lib.om_mg_level_size.argtypes = [C.c_void_p, C.c_int]
        lib.om_mg_parents.restype = C.POINTER(C.c_int)
        lib.om_mg_parents.argtypes = [C.c_void_p, C.c_int]
        lib.om_set_threads.restype = C.c_int
        lib.om_set_threads.argtypes = [C.c_int]
        lib.om_mg_width.restype = C.c_int
        lib.om_mg_width.argtypes = [C.c_void_p, C.c_int]
        lib.om_mg_coarse_matrix.restype = C.c_int
        lib.om_mg_coarse_matrix.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib = lib
    return _lib


def set_threads(n: int) -> int:
    """Threads of the AxOMP loop (the reference's OpenMP region); n <= 0 keeps
    the current count.  Returns the count in effect."""
    return load().om_set_threads(int(n))


class Oracle:
    """The sequential FP64 restatement for one mesh + case."""

    def __init__(self, mesh, case):
        from flowsolversourcecode_b200 import _lib as L
        self.lib = load()
        self._cfg = case.struct(mesh)
        ms, self._keep = L.mesh_struct(mesh)
        self.h = self.lib.om_create(C.byref(ms), C.byref(self._cfg))
        n, f, b, w = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        self.lib.om_sizes(self.h, C.byref(n), C.byref(f), C.byref(b), C.byref(w))
        self.N, self.F, self.B, self.W = n.value, f.value, b.value, w.value
        self.nIter = 0

    def arr(self, name: str) -> np.ndarray:
        """Live numpy view of an internal array (writes go to the oracle)."""
        ln, isint = C.c_long(), C.c_int()
        p = self.lib.om_array(self.h, name.encode(), C.byref(ln), C.byref(isint))
        if not p:
            raise KeyError(name)
        t = C.c_int32 if isint.value else C.c_double
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(t)), shape=(ln.value,))

    def get(self, name):
        return self.arr(name).copy()

    def set(self, name, values):
        self.arr(name)[:] = values

    def simple_iteration(self) -> float:
        self.nIter += 1
        return self.lib.om_simple_iteration(self.h)

    def momentum(self, comp: int):
        self.lib.om_momentum(self.h, comp)

    def assemble_momentum(self, comp: int):
        self.lib.om_assemble_momentum(self.h, comp)

    def continuity(self):
        self.lib.om_continuity(self.h)

    def assemble_continuity(self):
        self.lib.om_assemble_continuity(self.h)

    def correct_continuity(self):
        self.lib.om_correct_continuity(self.h)

    def set_iter(self, n: int):
        self.nIter = n
        self.lib.om_set_iter(self.h, n)

    def residuals(self) -> dict:
        a = (C.c_double * 20)()
        self.lib.om_residuals(self.h, a)
        a = list(a)
        return {"abs": a[0:5], "max": a[5:10], "rms": a[10:15], "scaled": a[15:20]}

    def residuals_turb(self) -> dict:
        """Residual norms of the k (index 0) and epsilon (index 1) equations."""
        a = (C.c_double * 8)()
        self.lib.om_residuals_turb(self.h, a)
        a = list(a)
        return {"abs": a[0:2], "max": a[2:4], "rms": a[4:6], "scaled": a[6:8]}

    def energy(self):
        """SolveEnergy ('temperature') on the current velocities and mdot."""
        self.lib.om_energy(self.h)

    def residuals_temp(self) -> dict:
        """Residual norms of the temperature equation (NF 6)."""
        a = (C.c_double * 4)()
        self.lib.om_residuals_temp(self.h, a)
        a = list(a)
        return {"abs": a[0], "max": a[1], "rms": a[2], "scaled": a[3]}

    def turb_production(self) -> np.ndarray:
        """k-epsilon production from the current gradients, k, epsilon, mu_t."""
        self.lib.om_turb_production(self.h)
        return self.get("prod")

    def initialize_mdot(self):
        """CalculateInitialmdot from the current velocity fields."""
        self.lib.om_initialize_mdot(self.h)

    def advance_time(self, dt_next: float):
        """Time-step prologue of the unsteady loop (MainProgram.for:184-245)."""
        self.lib.om_advance_time(self.h, float(dt_next))
        self.nIter = 0

    def adaptive_time_step(self, courant: float = 2.0, min_factor: float = 0.5, max_factor: float = 5.0) -> float:
        """AdaptiveTimeStep of a laminar, isothermal case (CalculateAdaptiveTimeStep.for:4-200):
        the next dt from the current mass fluxes, clamped to [min_factor dt, max_factor dt]."""
        return self.lib.om_adaptive_dt(self.h, float(courant), float(min_factor), float(max_factor))

    def get_time(self) -> dict:
        t = (C.c_double * 4)()
        n = C.c_int(0)
        self.lib.om_get_time(self.h, t, C.byref(n))
        return {"time": t[0], "dt": t[1], "dt_old": t[2], "dt_oldold": t[3], "ndt": n.value}

    def set_time(self, time: float, dt: float, dt_old: float, dt_oldold: float, ndt: int):
        t = (C.c_double * 4)(time, dt, dt_old, dt_oldold)
        self.lib.om_set_time(self.h, t, int(ndt))

    def lin_iters(self, nf: int) -> int:
        return self.lib.om_lin_iters(self.h, nf)

    def gradient(self, var: int, method: int, niter: int, phi, bphi):
        phi = np.ascontiguousarray(phi, np.float64)
        bphi = np.ascontiguousarray(bphi, np.float64)
        g = np.zeros(3 * self.N)
        bg = np.zeros(3 * self.B)
        self.lib.om_gradient(self.h, var, method, niter, phi.ctypes.data, bphi.ctypes.data, g.ctypes.data,
                             bg.ctypes.data)
        return g, bg

    def bicgstab(self, maxit=100, tol=1e-5) -> int:
        return self.lib.om_bicgstab(self.h, maxit, tol)

    def gmres(self) -> int:
        """GMRES_RESTARTED_OMP_RETURNR on the current system; dphi holds x."""
        return self.lib.om_gmres(self.h)

    def mg_setup(self) -> int:
        return self.lib.om_mg_setup(self.h)

    def mg_parents(self, level: int) -> np.ndarray:
        n = self.lib.om_mg_level_size(self.h, level)
        p = self.lib.om_mg_parents(self.h, level)
        return np.ctypeslib.as_array(p, shape=(n,)).copy()

    def mg_coarse_matrix(self, level: int) -> dict:
        """AssembleAgglomeratedLHS of the current system: the matrix of `level`."""
        n, w = self.lib.om_mg_level_size(self.h, level), self.lib.om_mg_width(self.h, level)
        out = {"ac": np.zeros(n), "n_nbr": np.zeros(n, np.int32), "nbr": np.zeros(n * w, np.int32),
               "anb": np.zeros(n * w)}
        rc = self.lib.om_mg_coarse_matrix(self.h, level, *[out[k].ctypes.data for k in ("ac", "n_nbr", "nbr", "anb")])
        if rc != 0:
            raise ValueError(f"no coarse level {level}")
        return out

    def close(self):
        if self.h:
            self.lib.om_destroy(self.h)
            self.h = None
