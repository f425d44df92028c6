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
from .mesh import BFS_PATCHES, BOX_PATCHES, PolyMesh, bfs_mesh, box_mesh, uniform01


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
    # patches: name -> (type, (u,v,w)); type "pressure_outlet" takes (type, static pressure),
    # "mass_inlet" ('specifiedmassflowrate') takes (type, (direction x,y,z), mass flow into the domain),
    # "pressure_inlet" ('specifiedstaticpressure' inlet) takes (type, (direction x,y,z), static pressure),
    # "mass_outlet" ('specifiedmassflowrate' outlet) takes (type, mass flow out of the domain),
    # "average_pressure_outlet" ('specifiedaveragestaticpressure') takes (type, average static pressure),
    # "resistance_outlet" ('specifiedresistance') takes (type, resistance, initial static pressure),
    # "stagnation_inlet" ('specifiedstagnationpressure') takes (type, (direction x,y,z), stagnation pressure)
    patches: dict = field(default_factory=dict)
    # 'fullydeveloped' outlets: patch name -> MassFlowFraction (default 1)
    mass_flow_fraction: dict = field(default_factory=dict)
    # k-epsilon (TurbulenceModel='kepsilon', equilibrium 'standard' wall functions)
    turbulence: bool = False
    solver_turb: str = "sor"               # ASSolverTKE = ASSolverTED
    rrf_tke: float = 0.1                   # rrfTKE
    rrf_ted: float = 0.1                   # rrfTED
    itmax_tke: int = 10                    # ASIterTKE
    itmax_ted: int = 3                     # ASIterTED
    urf_tke: float = 0.5                   # urfTKE
    urf_ted: float = 0.5                   # urfTED
    urf_tvisc: float = 0.5                 # urfTViscosity
    max_visc_ratio: float = 1.0e6          # MaximumViscosityRatio
    limit_production: bool = True          # LimitTurbulenceProduction
    conv_scheme_tke: str = "upwind"        # ConvectionSchemeTKE
    conv_scheme_ted: str = "minmod"        # ConvectionSchemeTED
    wall_function: str = "standard"        # MomentumWallFunctionType: 'standard' or 'scalable'
    # inlet patch name -> (inletTurbulenceIntensity, inletTurbulenceLengthScale), 'specifiedil'
    inlet_turbulence: dict = field(default_factory=dict)
    # unsteady runs (LUnsteady, TransientScheme, dt); time steps through Solver.advance_time
    unsteady: bool = False
    transient_scheme: str = "euler"        # 'euler', 'cranknicolson1', 'cranknicolson2', 'adamsmoulton'
    dt: float = 1.0e-2
    # temperature equation (LSolveEnergy, EnergyEquation='temperature'); defaults
    # of ProblemDescriptionRoutine.for:101-525 and User0.F90:83
    energy: bool = False
    cp: float = 1.0                        # SpecificHeat
    conductivity: float = 0.01             # Conductivity
    temp_init: float = 0.0                 # initial temperature
    solver_energy: str = "sor"             # ASSolverEnergy
    rrf_energy: float = 0.01               # rrfEnergy
    itmax_energy: int = 30                 # ASIterEnergy
    relax_energy: bool = True              # LRelaxEnergy
    urf_energy: float = 0.7                # urfEnergy
    conv_scheme_energy: str = "minmod"     # ConvectionSchemeEnergy
    bleed_energy: float = 0.0              # BleedEnergy
    method_grad_energy: int = 2            # MethodCalcGradientEnergy
    niter_grad_energy: int = 2             # nIterGradientEnergy
    grad_interp_energy: str = "average"    # GradientInterpolationSchemeEnergy
    gamma_interp_energy: str = "harmonic"  # InterpolationSchemeGamaEnergy
    energy_sc: float = 0.0                 # ScEnergy (uniform)
    energy_sb: float = 0.0                 # SbEnergy (uniform)
    limit_temperature: bool = False        # LimitTemperature
    temp_min: float = 0.0                  # tempmin
    temp_max: float = 1.0e30               # tempmax
    sigma_t: float = 0.0                   # SigT (0: the k-epsilon default 0.9)
    energy_wall_function: str = "standard" # EnergyWallFunctionType
    # patch name -> (thermal type, value[, h_inf]): "dirichlet" (T_wall), "vonneumann"
    # (heat flux), "robin" (T_inf, h_inf), "statictemperature" (T), "stagnationtemperature"
    # (T0), "fullydevelopedenergy", "symmetry"; unnamed patches take the flow type's default
    thermal: dict = field(default_factory=dict)
    # p' initial guess: least-squares combination of this many previous p'
    # solutions (AMG-BiCGSTAB solvers; no reference counterpart, 0 = zero start)
    pc_history: int = 0
    # rebuild the AMG preconditioner's coarse levels every this many p' solves (1: every solve)
    pc_refresh: int = 1

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
               "inlet": L.BC_INLET_VEL, "outlet": L.BC_OUTLET_FD, "pressure_outlet": L.BC_OUTLET_SP,
               "mass_inlet": L.BC_INLET_MASS, "pressure_inlet": L.BC_INLET_SP, "mass_outlet": L.BC_OUTLET_MASS,
               "average_pressure_outlet": L.BC_OUTLET_ASP, "resistance_outlet": L.BC_OUTLET_RES,
               "stagnation_inlet": L.BC_INLET_STAG}
        for s, name in enumerate(mesh.patch_names):
            spec = self.patches.get(name, ("wall", (0.0, 0.0, 0.0)))
            t, vel = spec[0], spec[1]
            c.patch_type[s] = bct[t]
            if t in ("pressure_outlet", "average_pressure_outlet"):   # (type, static | average static pressure)
                c.patch_pressure[s] = float(vel)
            elif t == "mass_outlet":     # (type, mass flow)
                c.patch_mass_flow[s] = float(vel)
            elif t == "resistance_outlet":   # (type, resistance, initial static pressure)
                c.patch_resistance[s] = float(vel)
                c.patch_pressure[s] = float(spec[2])
            elif t in ("mass_inlet", "pressure_inlet", "stagnation_inlet"):
                # (type, direction, mass flow | static pressure | stagnation pressure)
                for q in range(3):
                    c.patch_vel[s][q] = float(vel[q])
                if t == "mass_inlet":
                    c.patch_mass_flow[s] = float(spec[2])
                else:
                    c.patch_pressure[s] = float(spec[2])
            else:
                for q in range(3):
                    c.patch_vel[s][q] = float(vel[q])
            c.mass_flow_fraction[s] = float(self.mass_flow_fraction.get(name, 1.0))
            it, il = self.inlet_turbulence.get(name, (0.0, 1.0))
            c.inlet_intensity[s], c.inlet_length[s] = float(it), float(il)
        c.turbulence = int(self.turbulence)
        c.solver_turb = L.SOLVER[self.solver_turb]
        c.rrf_tke, c.rrf_ted = self.rrf_tke, self.rrf_ted
        c.itmax_tke, c.itmax_ted = self.itmax_tke, self.itmax_ted
        c.urf_tke, c.urf_ted, c.urf_tvisc = self.urf_tke, self.urf_ted, self.urf_tvisc
        c.max_visc_ratio, c.limit_production = self.max_visc_ratio, int(self.limit_production)
        c.conv_scheme_tke, c.conv_scheme_ted = L.TVD[self.conv_scheme_tke], L.TVD[self.conv_scheme_ted]
        c.wall_function = {"standard": 0, "scalable": 1, "automatic": 2}[self.wall_function]
        c.unsteady, c.transient_scheme, c.dt = int(self.unsteady), L.TRANSIENT[self.transient_scheme], float(self.dt)
        c.energy, c.cp, c.conductivity, c.temp_init = int(self.energy), self.cp, self.conductivity, self.temp_init
        c.solver_energy, c.rrf_energy, c.itmax_energy = L.SOLVER[self.solver_energy], self.rrf_energy, self.itmax_energy
        c.relax_energy, c.urf_energy = int(self.relax_energy), self.urf_energy
        c.conv_scheme_energy, c.bleed_energy = L.TVD[self.conv_scheme_energy], self.bleed_energy
        c.method_grad_energy, c.niter_grad_energy = self.method_grad_energy, self.niter_grad_energy
        c.grad_interp_energy = gi[self.grad_interp_energy]
        c.gamma_interp_energy = {"average": 0, "upwind": 1, "downwind": 2, "harmonic": 3}[self.gamma_interp_energy]
        c.energy_sc, c.energy_sb = self.energy_sc, self.energy_sb
        c.limit_temperature, c.temp_min, c.temp_max = int(self.limit_temperature), self.temp_min, self.temp_max
        c.sigma_t = self.sigma_t
        c.energy_wall_function = {"standard": 0, "scalable": 1, "automatic": 2}[self.energy_wall_function]
        c.pc_history = int(self.pc_history)
        c.pc_refresh = int(self.pc_refresh)
        for s, name in enumerate(mesh.patch_names):
            spec = self.thermal.get(name, ("default",))
            c.patch_thermal[s] = L.TBC[spec[0]]
            if spec[0] == "vonneumann":
                c.patch_heat_flux[s] = float(spec[1])
            elif spec[0] == "robin":
                c.patch_temperature[s], c.patch_h_inf[s] = float(spec[1]), float(spec[2])
            elif len(spec) > 1:
                c.patch_temperature[s] = float(spec[1])
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


def bfs(nx: int = 512, ny: int = 96, nz: int = 48, re_h: float = 5000.0, intensity: float = 0.05,
        length: float = 0.1, **kw) -> tuple[PolyMesh, Case]:
    """3-D backward-facing step, steady RANS k-epsilon with wall functions.

    Channel 30H x 3H x 2H (H = 1), step wall at x = 0 for y < H, inlet at
    x = 0 for y >= H with u = 1, outlet 'fullydeveloped' at x = 30H, no-slip
    walls elsewhere; rho = 1, mu = 1/Re_H.  Inlet turbulence 'specifiedil'
    with the given intensity and length scale.  Momentum wall functions
    'automatic' (the reference's default type) and the bounded minmod TVD
    scheme for momentum from iteration 1: with 'standard' wall functions or
    unbounded second-order upwind the outer iteration settles into a limit
    cycle instead of converging.  Use :func:`bfs_initial_state` for the
    initial fields (perturbed inlet profile)."""
    mesh = bfs_mesh(nx, ny, nz)
    patches = {p: ("wall", (0.0, 0.0, 0.0)) for p in BFS_PATCHES}
    patches["inlet"] = ("inlet", (1.0, 0.0, 0.0))
    patches["xmax"] = ("outlet", (0.0, 0.0, 0.0))
    kw.setdefault("conv_scheme", "minmod")
    kw.setdefault("niter_start_hr", 1)
    kw.setdefault("turbulence", True)
    kw.setdefault("wall_function", "automatic")
    case = Case(mu=1.0 / re_h, patches=patches, inlet_turbulence={"inlet": (intensity, length)}, **kw)
    return mesh, case


def bfs_initial_state(mesh: PolyMesh, case: Case, seed: int = 0, perturbation: float = 0.05) -> dict:
    """Initial fields of the step case: u = 1 in every cell and on the outlet,
    inlet faces u = 1 + perturbation * U(-1, 1) (splitmix64 from `seed`, one
    draw per inlet face in boundary order), k and epsilon uniform at the
    inlet-turbulence values of a unit velocity (k = 1.5 I^2, eps =
    Cmu^0.75 k^1.5 / L) and mu_t = Cmu rho k^2 / eps, on cells and boundary faces
    (turbulent cases only).  Apply with ``obj.set(name, value)`` for every item, then
    ``obj.initialize_mdot()``."""
    N = mesh.n_cells
    B = mesh.n_faces - mesh.n_internal
    F = mesh.n_internal
    s_in = mesh.patch("inlet")
    b0 = int(mesh.patch_start[s_in]) - F
    nin = int(mesh.patch_size[s_in])
    bu = np.zeros(B)
    s_out = mesh.patch("xmax")
    o0 = int(mesh.patch_start[s_out]) - F
    bu[o0:o0 + int(mesh.patch_size[s_out])] = 1.0
    bu[b0:b0 + nin] = 1.0 + perturbation * (2.0 * uniform01(seed, nin) - 1.0)
    it, ln = case.inlet_turbulence.get("inlet", (0.05, 0.1))
    k0 = 1.5 * 1.0 * it * it
    cmu = float(np.float32(0.09))
    cmu75 = np.sqrt(np.sqrt(cmu)) ** 3
    e0 = cmu75 * k0 ** 1.5 / ln
    mut0 = cmu * case.rho * k0 * k0 / e0
    state = {"u": np.ones(N), "bu": bu}
    if case.turbulence:
        state.update({"tke": np.full(N, k0), "ted": np.full(N, e0), "mut": np.full(N, mut0),
                      "btke": np.full(B, k0), "bted": np.full(B, e0), "bmut": np.full(B, mut0)})
    return state
