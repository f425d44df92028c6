"""Temperature equation (EnergyEquation='temperature',
Energy/SolveTemperatureEquation.for): the CPU restatement's analytic pins
(CPU) and the GPU path against it (gpu).

Pins: one-dimensional conduction between Dirichlet, von Neumann and Robin
walls has a linear exact solution that the finite-volume scheme reproduces on
a uniform box; a heated lid-driven cavity conserves energy at convergence;
the thermal wall function's diffusion coefficient follows the law of the wall
(WallFunctions.for:743-1005) from the momentum wall functions' uTau and y+."""

import numpy as np
import pytest

from flowsolversourcecode_b200 import case as cs
from flowsolversourcecode_b200 import mesh as fm


def _oracle(mesh, case):
    import oracle
    return oracle.Oracle(mesh, case)


def _patch_slice(mesh, name):
    s = mesh.patch(name)
    b0 = int(mesh.patch_start[s]) - mesh.n_internal
    return slice(b0, b0 + int(mesh.patch_size[s]))


def _conduction_case(thermal, k=0.5, **kw):
    """Still fluid in a closed box: the temperature equation is pure conduction
    (unrelaxed, so each outer iteration solves it to the Krylov tolerance)."""
    kw.setdefault("relax_energy", False)
    kw.setdefault("solver_energy", "bicgs")
    kw.setdefault("krylov_tol", 1e-14)
    kw.setdefault("krylov_maxit", 400)
    return cs.Case(rho=1.0, mu=0.01, energy=True, conductivity=k, cp=1.0, thermal=thermal,
                   patches={}, **kw)


def _run_energy(o, n):
    for _ in range(n):
        o.energy()


# ------------------------------------------------------------------- CPU
def test_conduction_dirichlet_linear_profile(oracle_lib):
    mesh = fm.box_mesh(8, 3, 2)
    case = _conduction_case({"xmin": ("dirichlet", 1.0), "xmax": ("dirichlet", 0.0)})
    o = _oracle(mesh, case)
    _run_energy(o, 4)
    xc = o.get("xc")
    assert np.max(np.abs(o.get("temp") - (1.0 - xc))) < 1e-10


def test_conduction_heat_flux_wall(oracle_lib):
    # heat q per unit area enters at x = 1 and leaves through the T = 0 wall: T = q x / k
    q, k = 2.0, 0.5
    mesh = fm.box_mesh(8, 3, 2)
    case = _conduction_case({"xmin": ("dirichlet", 0.0), "xmax": ("vonneumann", q)}, k=k)
    o = _oracle(mesh, case)
    _run_energy(o, 4)
    assert np.max(np.abs(o.get("temp") - q * o.get("xc") / k)) < 1e-10


def test_conduction_robin_wall(oracle_lib):
    # T(0) = 1, k T'(1) = -h (T(1) - Tinf): T = 1 + s x with s = h (Tinf - 1) / (k + h)
    k, h, tinf = 0.5, 2.0, 0.0
    mesh = fm.box_mesh(10, 2, 2)
    case = _conduction_case({"xmin": ("dirichlet", 1.0), "xmax": ("robin", tinf, h)}, k=k)
    o = _oracle(mesh, case)
    _run_energy(o, 4)
    s = h * (tinf - 1.0) / (k + h)
    assert np.max(np.abs(o.get("temp") - (1.0 + s * o.get("xc")))) < 1e-10
    # the Robin face temperature balances the two resistances
    bt = o.get("btemp")[_patch_slice(mesh, "xmax")]
    assert np.max(np.abs(bt - (1.0 + s))) < 1e-10


def test_uniform_temperature_stays_uniform_in_flow(oracle_lib):
    # inlet at the initial temperature, adiabatic walls: T stays uniform
    mesh, case = cs.bfs(12, 6, 4)
    case.energy, case.temp_init = True, 3.0
    case.thermal = {"inlet": ("statictemperature", 3.0)}
    o = _oracle(mesh, case)
    for k, v in cs.bfs_initial_state(mesh, case, seed=0, perturbation=0.0).items():
        o.set(k, v)
    o.initialize_mdot()
    for _ in range(3):
        o.simple_iteration()
    assert np.max(np.abs(o.get("temp") - 3.0)) < 1e-12
    assert abs(o.residuals_temp()["abs"]) < 1e-10


def test_heated_cavity_conserves_energy(oracle_lib):
    mesh, case = cs.cavity(8, nz=1, re=100.0)
    case.energy, case.conductivity, case.cp = True, 0.02, 1.0
    case.thermal = {"ymax": ("dirichlet", 1.0), "ymin": ("dirichlet", 0.0)}
    case.solver_energy = "bicgs"
    case.max_residual = 1e-9
    case.krylov_tol, case.krylov_maxit = 1e-13, 400
    case.solver_cont = "bicgs"
    o = _oracle(mesh, case)
    for _ in range(400):
        if o.simple_iteration() < case.max_residual:
            break
    t, bt, gd = o.get("temp"), o.get("btemp"), o.get("bgdiff")
    own = o.get("bf_own")
    q = case.conductivity * gd * (bt - t[own])       # conduction into the domain per face
    qin, qout = q[_patch_slice(mesh, "ymax")].sum(), q[_patch_slice(mesh, "ymin")].sum()
    assert qin > 0 > qout
    assert abs(qin + qout) < 1e-6 * qin
    assert np.all((t > 0.0) & (t < 1.0))


@pytest.mark.parametrize("kind", ["standard", "scalable", "automatic"])
def test_thermal_wall_function_coefficient(oracle_lib, kind):
    mesh, case = cs.bfs(16, 6, 4)
    case.energy, case.energy_wall_function = True, kind
    case.conductivity, case.cp = 1e-4, 1.0
    case.thermal = {"inlet": ("statictemperature", 1.0), "step": ("dirichlet", 2.0), "ymin": ("dirichlet", 2.0)}
    o = _oracle(mesh, case)
    for k, v in cs.bfs_initial_state(mesh, case, seed=0, perturbation=0.0).items():
        o.set(k, v)
    o.initialize_mdot()
    for _ in range(3):
        o.simple_iteration()
    f32 = lambda x: float(np.float32(x))
    pr = case.mu * case.cp / case.conductivity
    prp = (f32(3.85) * pr ** f32(1.0 / 3.0) - f32(1.3)) ** 2
    utau, yp, wd, bedif = o.get("utau"), o.get("yplus"), o.get("wdist"), o.get("bedif")
    own, bt = o.get("bf_own"), o.get("btype")
    walls = np.nonzero(bt == 0)[0]
    assert walls.size > 0
    for b in walls[::7]:
        pry = pr * yp[b]
        if kind == "scalable":
            pry = max(pry, f32(11.63))
            tp = f32(2.12) * np.log(pry) + prp
        elif kind == "automatic":
            g = f32(0.01) * pry ** 4 / (1 + 5 * pr * pr * pry) + 1e-15
            tp = pry * np.exp(-g) + (f32(2.12) * np.log(pry) + prp) * np.exp(-1 / g)
        else:
            tp = pry if pry < f32(11.63) else f32(2.12) * np.log(pry) + prp
        wvt = utau[b] * case.rho * case.cp * wd[own[b]] / max(tp, 1e-15)
        ref = max(wvt, case.conductivity)
        assert abs(bedif[b] - ref) <= 1e-12 * ref, (b, bedif[b], ref)


# ------------------------------------------------------------------- GPU
def _tight(**kw):
    kw.setdefault("solver_mom", "bicgs")
    kw.setdefault("solver_cont", "bicgs")
    kw.setdefault("solver_energy", "bicgs")
    kw.setdefault("krylov_tol", 1e-13)
    kw.setdefault("krylov_maxit", 400)
    return kw


def _compare(s, o, names, tol):
    for k in names:
        g, r = s.get(k), o.get(k)
        err = np.max(np.abs(g - r)) / max(np.max(np.abs(r)), 1e-30)
        assert err <= tol, (k, err)


def _heated_cavity(n=10, **kw):
    mesh, case = cs.cavity(n, nz=3, re=100.0, jitter=0.15, seed=3)
    kw = _tight(**kw)
    for k, v in kw.items():
        setattr(case, k, v)
    case.energy, case.conductivity, case.cp = True, 0.02, 1.3
    case.conv_scheme_energy = "minmod"
    case.niter_start_hr = 1
    case.thermal = {"ymax": ("dirichlet", 1.0), "ymin": ("robin", 0.2, 3.0), "xmin": ("vonneumann", 0.5)}
    return mesh, case


@pytest.mark.gpu
def test_energy_cavity_iterations_match_oracle():
    from flowsolversourcecode_b200.solver import Solver
    mesh, case = _heated_cavity()
    s, o = Solver(mesh, case), _oracle(mesh, case)
    for it in range(6):
        rg = s.simple_iteration()
        so = o.simple_iteration()
        ro = o.residuals_temp()
        assert abs(rg["temp_abs"] - ro["abs"]) <= 1e-9 * abs(ro["abs"]) + 1e-14, (it, rg["temp_abs"], ro["abs"])
        assert abs(rg["source"] - so) <= 1e-6 * abs(so) + 1e-14, (it, rg["source"], so)
    _compare(s, o, [("temp"), ("btemp")], 1e-9)


@pytest.mark.gpu
def test_energy_assembly_bit_level():
    """One temperature assembly on the same state: ac, anb, bc at 1e-14."""
    from flowsolversourcecode_b200.solver import Solver
    mesh, case = _heated_cavity(n=8)
    case.itmax_energy, case.solver_energy = 0, "sor"
    s, o = Solver(mesh, case), _oracle(mesh, case)
    rng = np.random.default_rng(5)
    st = {"u": rng.uniform(-1, 1, s.N), "v": rng.uniform(-1, 1, s.N), "w": rng.uniform(-0.2, 0.2, s.N),
          "temp": rng.uniform(0, 1, s.N)}
    for k, v in st.items():
        s.set(k, v)
        o.set(k, v)
    s.initialize_mdot()
    o.initialize_mdot()
    s.set_iteration(5)
    o.set_iter(5)
    s.energy()
    o.energy()
    for k in ("ac", "bc"):
        g, r = s.get(k), o.get(k)
        assert np.max(np.abs(g - r)) <= 1e-14 * np.max(np.abs(r)), k
    W = s.W
    g = s.get("anb").reshape(W, -1)
    r = o.get("anb").reshape(W, -1)
    assert np.max(np.abs(g - r)) <= 1e-14 * np.max(np.abs(r))


@pytest.mark.gpu
@pytest.mark.parametrize("wf", ["standard", "automatic"])
def test_energy_kepsilon_step_matches_oracle(wf):
    from flowsolversourcecode_b200.solver import Solver
    mesh, case = cs.bfs(24, 6, 4)
    for k, v in _tight(solver_turb="bicgs").items():
        setattr(case, k, v)
    case.energy, case.energy_wall_function = True, wf
    case.conductivity, case.cp = 2e-4, 1.0
    case.thermal = {"inlet": ("statictemperature", 1.0), "step": ("dirichlet", 2.0),
                    "ymin": ("vonneumann", 0.01), "ymax": ("robin", 0.5, 0.3)}
    s, o = Solver(mesh, case), _oracle(mesh, case)
    for k, v in cs.bfs_initial_state(mesh, case, seed=0, perturbation=0.0).items():
        s.set(k, v)
        o.set(k, v)
    s.initialize_mdot()
    o.initialize_mdot()
    for it in range(4):
        rg = s.simple_iteration()
        o.simple_iteration()
        ro = o.residuals_temp()
        assert abs(rg["temp_abs"] - ro["abs"]) <= 1e-8 * abs(ro["abs"]) + 1e-14, (it, rg["temp_abs"], ro["abs"])
    _compare(s, o, ["temp", "btemp"], 1e-8)


@pytest.mark.gpu
def test_energy_stagnation_inlet_transient_matches_oracle():
    from flowsolversourcecode_b200.solver import Solver
    mesh, case = cs.bfs(18, 6, 4)
    case.turbulence = False
    for k, v in _tight().items():
        setattr(case, k, v)
    case.unsteady, case.transient_scheme, case.dt = True, "cranknicolson2", 0.05
    case.energy, case.conductivity, case.cp = True, 1e-3, 2.0
    case.energy_sc, case.energy_sb = -0.1, 0.3
    case.thermal = {"inlet": ("stagnationtemperature", 1.5), "step": ("dirichlet", 2.0)}
    case.limit_temperature, case.temp_min, case.temp_max = True, 0.0, 1.9
    s, o = Solver(mesh, case), _oracle(mesh, case)
    for k, v in cs.bfs_initial_state(mesh, case, seed=0, perturbation=0.0).items():
        s.set(k, v)
        o.set(k, v)
    s.initialize_mdot()
    o.initialize_mdot()
    for step in range(3):
        s.advance_time(0.05)
        o.advance_time(0.05)
        for it in range(3):
            rg = s.simple_iteration()
            o.simple_iteration()
            ro = o.residuals_temp()
            assert abs(rg["temp_abs"] - ro["abs"]) <= 1e-8 * abs(ro["abs"]) + 1e-14, (step, it)
    _compare(s, o, ["temp", "btemp", "old"], 1e-8)
