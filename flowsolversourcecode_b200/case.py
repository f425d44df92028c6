"""Case descriptions: the knobs of the reference's User0 module and
DescribeProblem entries (ProblemDesciption/ProblemDescriptionRoutine.for:201-524)
that the SIMPLE inner loop reads, plus the synthetic benchmark cases.

A reference DescribeProblem that assigns a default-real literal to a double
knob (e.g. ``urfMomentum=0.7``) stores the REAL(4)-rounded value;
:func:`ref_real` reproduces that rounding for users who want bit-level
agreement with such a case file.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from . import _lib as L
from .mesh import BOX_PATCHES, PolyMesh, box_mesh


def ref_real(x: float) -> float:
    """Value a default-real (REAL(4)) Fortran literal has once stored in a double."""
    return float(np.float32(x))


@dataclass
class Case:
    # physics
    rho: float = 1.0
    mu: float = 0.01
    algorithm: str = "simplec"             # Algorithm (the shipped case's 'simplec')
    # under-relaxation
    relax_momentum: bool = True            # LRelaxMomentum
    urf_momentum: float = 0.7              # urfMomentum
    urf_pressure: float = 0.7              # urfPressure
    # gradients (User0.F90:98-160)
    method_grad_mom: int = 2
    method_grad_cont: int = 2
    niter_grad_mom: int = 2
    niter_grad_cont: int = 2
    grad_interp_mom: str = "average"
    grad_interp_cont: str = "averagecorrected"
    method_decompose_s: int = 3            # MethodDecomposeS
    # convection
    hr_framework: str = "tvd"
    conv_scheme: str = "upwind"            # ConvectionSchemeMomentum
    niter_start_hr: int = 10000            # nIterStartApplyingHR
    bleed: float = 0.0
    # algebraic solvers
    solver_mom: str = "sor"
    solver_cont: str = "bicgs"
    rrf_mom: float = 0.01
    rrf_cont: float = 0.001
    itmax_mom: int = 30
    itmax_cont: int = 100
    krylov_maxit: int = 100                # BICGSTAB_OMP(N,100,1.d-5)
    krylov_tol: float = 1.0e-5
    # stop criterion
    nstop_type: int = 4
    max_residual: float = 1.0e-6
    ref_pressure_cell: int = 0             # ReferencePressureLocation=1 (0-based here)
    set_reference_pressure: int = -1       # computed (no pressure-specified patch types)
    inviscid: bool = False
    # multigrid
    mg_cycle: str = "v"
    mg_pre: int = 1
    mg_post: int = 3
    mg_max_cycles: int = 30
    mg_min_parents: int = 10
    mg_max_levels: int = 10
    mg_rrf: float = 0.1
    # multi-RHS momentum (X, Y, Z solved together; no reference counterpart)
    batched_momentum: bool = False
    # patches: name -> (type, (u,v,w))
    patches: dict = field(default_factory=dict)

    def struct(self, mesh: PolyMesh) -> L.FsCase:
        c = L.FsCase()
        c.rho, c.mu = self.rho, self.mu
        c.algorithm = L.SIMPLE if self.algorithm == "simple" else L.SIMPLEC
        c.relax_momentum = int(self.relax_momentum)
        c.urf_momentum, c.urf_pressure = self.urf_momentum, self.urf_pressure
        c.method_grad_mom, c.method_grad_cont = self.method_grad_mom, self.method_grad_cont
        c.niter_grad_mom, c.niter_grad_cont = self.niter_grad_mom, self.niter_grad_cont
        gi = {"average": L.GI_AVERAGE, "upwind": L.GI_UPWIND, "downwind": L.GI_DOWNWIND,
              "averagecorrected": L.GI_AVERAGECORRECTED}
        c.grad_interp_mom, c.grad_interp_cont = gi[self.grad_interp_mom], gi[self.grad_interp_cont]
        c.method_decompose_s = self.method_decompose_s
        c.hr_framework = L.HR_TVD if self.hr_framework == "tvd" else L.HR_NONE
        c.conv_scheme = L.TVD[self.conv_scheme]
        c.niter_start_hr, c.bleed = self.niter_start_hr, self.bleed
        c.solver_mom, c.solver_cont = L.SOLVER[self.solver_mom], L.SOLVER[self.solver_cont]
        c.rrf_mom, c.rrf_cont = self.rrf_mom, self.rrf_cont
        c.itmax_mom, c.itmax_cont = self.itmax_mom, self.itmax_cont
        c.nstop_type, c.max_residual = self.nstop_type, self.max_residual
        c.ref_pressure_cell = self.ref_pressure_cell
        c.set_reference_pressure = self.set_reference_pressure
        c.inviscid = int(self.inviscid)
        c.mg_cycle = {"v": 0, "f": 1, "w": 2}[self.mg_cycle]
        c.mg_pre, c.mg_post, c.mg_max_cycles = self.mg_pre, self.mg_post, self.mg_max_cycles
        c.mg_min_parents, c.mg_max_levels, c.mg_rrf = self.mg_min_parents, self.mg_max_levels, self.mg_rrf
        c.krylov_maxit, c.krylov_tol = self.krylov_maxit, self.krylov_tol
        c.batched_momentum = int(self.batched_momentum)
        c.n_patches = len(mesh.patch_names)
        bct = {"wall": L.BC_WALL_NOSLIP, "slip": L.BC_WALL_SLIP, "symmetry": L.BC_SYMMETRY,
               "inlet": L.BC_INLET_VEL, "outlet": L.BC_OUTLET_FD}
        for s, name in enumerate(mesh.patch_names):
            t, vel = self.patches.get(name, ("wall", (0.0, 0.0, 0.0)))
            c.patch_type[s] = bct[t]
            for q in range(3):
                c.patch_vel[s][q] = float(vel[q])
        return c


def cavity(n: int, nz: int | None = None, re: float = 100.0, lid: float = 1.0, jitter: float = 0.0,
           seed: int = 0, **kw) -> tuple[PolyMesh, Case]:
    """Lid-driven cavity on the unit square/cube, lid = ymax moving in +x.

    nz=1 gives the 2-D cavity (one cell thick, z patches symmetry); otherwise
    an n^3 cube with all walls no-slip.  mu = lid*1/Re with rho=1.
    """
    if nz == 1:
        mesh = box_mesh(n, n, 1, 1.0, 1.0, 1.0 / n, jitter=jitter, seed=seed)
    else:
        nz = n if nz is None else nz
        mesh = box_mesh(n, n, nz, 1.0, 1.0, 1.0, jitter=jitter, seed=seed)
    patches = {p: ("wall", (0.0, 0.0, 0.0)) for p in BOX_PATCHES}
    patches["ymax"] = ("wall", (lid, 0.0, 0.0))
    if nz == 1:
        patches["zmin"] = ("symmetry", (0.0, 0.0, 0.0))
        patches["zmax"] = ("symmetry", (0.0, 0.0, 0.0))
    case = Case(mu=lid * 1.0 / re, patches=patches, **kw)
    return mesh, case


def cavity2d_64(**kw):
    """64x64x1 cavity, Re=100, upwind, SIMPLEC, urf 0.7/0.7 (the CPU-runnable case)."""
    return cavity(64, nz=1, re=100.0, **kw)


def cavity3d(n: int = 128, **kw):
    """n^3 cavity, Re=1000, second-order upwind deferred correction from iteration 1."""
    kw.setdefault("conv_scheme", "sou")
    kw.setdefault("niter_start_hr", 1)
    return cavity(n, re=1000.0, **kw)


def cavity3d_distorted(n: int = 128, seed: int = 0, **kw):
    """n^3 cavity with interior nodes jittered by U(-0.2h, 0.2h) from `seed`."""
    kw.setdefault("conv_scheme", "sou")
    kw.setdefault("niter_start_hr", 1)
    return cavity(n, re=1000.0, jitter=0.2, seed=seed, **kw)
