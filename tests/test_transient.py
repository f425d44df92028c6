"""Unsteady runs: the transient term of AssembleTheTransientTerm.for for the
four TransientScheme values, the time-step prologue of MainProgram.for:184-245
(first step of the three-level schemes as 'euler', the Crank-Nicolson
extrapolation, updateVariablesInTime, dt bookkeeping) and restarts from the
old time levels.  CPU tests pin the restatement; gpu tests hold the device
time stepping to it."""

import numpy as np
import pytest

from flowsolversourcecode_b200 import case as cs

SCHEMES = ["euler", "cranknicolson1", "cranknicolson2", "adamsmoulton"]
STATE = ("u", "v", "w", "p", "mdot", "bu", "bv", "bw", "bp", "bmdot")


def _cavity(scheme, dt=0.05, **kw):
    kw.setdefault("solver_mom", "bicgs")
    kw.setdefault("solver_cont", "bicgs")
    kw.setdefault("krylov_tol", 1e-13)
    kw.setdefault("krylov_maxit", 400)
    return cs.cavity(8, nz=6, jitter=0.2, seed=0, conv_scheme="sou", niter_start_hr=1,
                     unsteady=True, transient_scheme=scheme, dt=dt, **kw)


def _seed(obj, n, seed):
    rng = np.random.default_rng(seed)
    for k in ("u", "v", "w", "p"):
        obj.set(k, 0.05 * rng.standard_normal(n))


def _factors(scheme, dt, dto, dtoo):
    """(c1, c2, c3) with FluxCE = c1 rho V, FluxTE += rho V (c1 phi + c2 phiOld + c3 phiOldOld)."""
    if scheme == "euler":
        return 1 / dt, -1 / dt, 0.0
    if scheme == "cranknicolson1":
        return 2 / dt, -2 / dt, 0.0
    if scheme == "cranknicolson2":
        return ((dto / dt) / (dt + dto), 1 / (dt + dto) - (dtoo / dt) / (dto + dtoo),
                -(dto / dt) / (dto + dtoo))
    f1 = 1 / dt + 1 / (dt + dto)
    f3 = (dto / dt) / (dto + dtoo)
    return f1, -(f1 + f3), f3


# ------------------------------------------------------------------- CPU
@pytest.mark.parametrize("scheme", SCHEMES)
def test_oracle_transient_term(scheme):
    """ac and bc of an unsteady X-momentum assembly differ from the steady
    one on the same state by exactly the transient term."""
    import oracle
    m, c = _cavity(scheme, dt=0.05)
    cst = _cavity("euler")[1]
    cst.unsteady = False
    o = oracle.Oracle(m, c)
    s = oracle.Oracle(m, cst)
    N = o.N
    _seed(o, N, 1)
    o.simple_iteration()          # 'cranknicolson1' re-assembles mdot from D and gradients of an iteration
    o.advance_time(0.05)
    _seed(o, N, 2)
    o.simple_iteration()
    o.advance_time(0.04)          # dt changes: dtOld = dtOldOld = 0.05, dt = 0.04
    _seed(o, N, 3)
    t = o.get_time()
    assert t["ndt"] == 2 and t["dt"] == 0.04 and t["dt_old"] == 0.05 and t["dt_oldold"] == 0.05
    assert t["time"] == 0.05 + 0.04   # time += dt after dt = dt_next (MainProgram.for:236-244)
    for k in STATE:
        s.set(k, o.get(k))
    for obj in (o, s):
        obj.set_iter(1)
        obj.assemble_momentum(0)
    c1, c2, c3 = _factors(scheme, 0.04, 0.05, 0.05)
    V, u = o.get("vol"), o.get("u")
    uo, uoo = o.get("old")[:N], o.get("oldold")[:N]
    dac = (o.get("ac") - s.get("ac")) * c.urf_momentum
    np.testing.assert_allclose(dac, c1 * c.rho * V, rtol=1e-9)
    dbc = o.get("bc") - s.get("bc")
    want = -(c.rho * V * (c1 * u + c2 * uo + c3 * uoo))
    assert np.abs(dbc - want).max() <= 1e-9 * np.abs(want).max()


def test_oracle_three_level_schemes_start_with_euler():
    import oracle
    runs = {}
    for scheme in ("euler", "cranknicolson2", "adamsmoulton"):
        m, c = _cavity(scheme)
        o = oracle.Oracle(m, c)
        _seed(o, o.N, 5)
        out = []
        for step in range(2):
            o.advance_time(0.05)
            for _ in range(3):
                o.simple_iteration()
            out.append(o.get("u").copy())
        runs[scheme] = out
    for scheme in ("cranknicolson2", "adamsmoulton"):
        assert np.array_equal(runs[scheme][0], runs["euler"][0]), scheme
        assert not np.array_equal(runs[scheme][1], runs["euler"][1]), scheme


def test_oracle_crank_nicolson_extrapolates():
    """From the second step on 'cranknicolson1' starts from 2 phi - phiOld."""
    import oracle
    m, c = _cavity("cranknicolson1")
    o = oracle.Oracle(m, c)
    _seed(o, o.N, 6)
    o.advance_time(0.05)
    for _ in range(2):
        o.simple_iteration()
    u1, old = o.get("u"), o.get("old")[: o.N]
    o.advance_time(0.05)
    np.testing.assert_array_equal(o.get("u"), 2.0 * u1 - old)
    np.testing.assert_array_equal(o.get("old")[: o.N], 2.0 * u1 - old)


def test_oracle_unsteady_cavity_stationary_state():
    """Marched to a stationary state, an unsteady cavity differs from the
    steady solution only through D = V/ac in the Rhie-Chow flux (ac holds
    rho V c1; the transient Rhie-Chow correction adds 0 in the reference), so
    the difference scales with c1: x0.1 for a 10x larger dt, x1.5 for
    'adamsmoulton' (c1 = 1.5/dt) against 'euler' (c1 = 1/dt)."""
    import oracle
    mesh, c = cs.cavity(12, nz=1, solver_mom="bicgs", solver_cont="bicgs", krylov_tol=1e-12, krylov_maxit=300)
    st = oracle.Oracle(mesh, c)
    for _ in range(2000):
        if st.simple_iteration() < 1e-10:
            break
    ref = st.get("u")
    errs = {}
    for scheme, dt in (("euler", 2.0), ("euler", 20.0), ("adamsmoulton", 2.0)):
        c.unsteady, c.transient_scheme, c.dt = True, scheme, dt
        o = oracle.Oracle(mesh, c)
        prev = o.get("u")
        for step in range(40):
            o.advance_time(dt)
            for _ in range(60):
                if o.simple_iteration() < 1e-9:
                    break
            u = o.get("u")
            change, prev = np.abs(u - prev).max(), u
            if change < 1e-8:
                break
        assert change < 1e-8, (scheme, dt, change)
        assert o.get_time()["ndt"] == step + 1
        errs[scheme, dt] = np.abs(u - ref).max() / np.abs(ref).max()
    assert 5e-4 < errs["euler", 2.0] < 2e-2, errs
    assert 0.07 < errs["euler", 20.0] / errs["euler", 2.0] < 0.14, errs
    assert 1.3 < errs["adamsmoulton", 2.0] / errs["euler", 2.0] < 1.7, errs


# ------------------------------------------------------------------- GPU
def _pair(scheme, mesh_case=None, seed=4):
    import oracle
    from flowsolversourcecode_b200.solver import Solver
    m, c = mesh_case or _cavity(scheme)
    o = oracle.Oracle(m, c)
    g = Solver(m, c)
    if c.turbulence:
        for k, v in cs.bfs_initial_state(m, c, seed=seed).items():
            o.set(k, v)
            g.set(k, v)
        o.initialize_mdot()
        g.initialize_mdot()
    else:
        rng = np.random.default_rng(seed)
        for k in ("u", "v", "w", "p"):
            x = 0.05 * rng.standard_normal(o.N)
            o.set(k, x)
            g.set(k, x)
    return o, g


def _rel(x, ref):
    return float(np.linalg.norm(x - ref) / max(np.linalg.norm(ref), 1e-300))


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", SCHEMES)
def test_transient_assembly_matches_oracle(scheme):
    """The transient term itself: the X-momentum system after two time steps
    agrees with the restatement to round-off."""
    o, g = _pair(scheme)
    for step, dt in enumerate((0.05, 0.04)):
        o.simple_iteration()
        g.simple_iteration()
        o.advance_time(dt)
        g.advance_time(dt)
        for obj in (o, g):
            _seed(obj, o.N, 10 + step)
    for k in STATE:
        assert _rel(g.get(k), o.get(k)) <= 1e-14, k
    o.set_iter(1)
    g.set_iteration(1)
    o.assemble_momentum(0)
    g.assemble_momentum(0)
    for k in ("ac", "bc", "anb"):
        assert _rel(g.get(k), o.get(k)) <= 1e-14, k
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", SCHEMES)
def test_transient_steps_match_oracle(scheme):
    o, g = _pair(scheme)
    for step in range(3):
        o.advance_time(0.05)
        g.advance_time(0.05)
        for it in range(3):
            so = o.simple_iteration()
            rg = g.simple_iteration()
            assert abs(rg["source"] - so) <= 1e-6 * abs(so) + 1e-14, (step, it, rg["source"], so)
    for k in STATE + ("old", "oldold"):
        assert _rel(g.get(k), o.get(k)) <= 1e-8, k
    tg, to = g.time_state(), o.get_time()
    assert tg == to
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", ["euler", "cranknicolson1"])
def test_transient_kepsilon_step_matches_oracle(scheme):
    mc = cs.bfs(24, 9, 6, solver_mom="bicgs", solver_cont="bicgs", solver_turb="bicgs", krylov_tol=1e-13,
                krylov_maxit=400, unsteady=True, transient_scheme=scheme, dt=0.02)
    o, g = _pair(scheme, mc)
    for step in range(3):
        o.advance_time(0.02)
        g.advance_time(0.02)
        for it in range(3):
            so = o.simple_iteration()
            rg = g.simple_iteration()
            assert abs(rg["source"] - so) <= 1e-6 * abs(so) + 1e-14, (step, it)
    for k in ("u", "v", "w", "p", "tke", "ted", "mut", "bmdot", "old", "oldold", "bold"):
        assert _rel(g.get(k), o.get(k)) <= 1e-8, k
    g.close()


@pytest.mark.gpu
def test_unsteady_restart_continues_bitwise(tmp_path):
    from flowsolversourcecode_b200.solver import Solver
    m, c = _cavity("adamsmoulton")
    runs = []
    for restart in (False, True):
        g = Solver(m, c)
        _seed(g, g.N, 8)
        for step in range(4):
            if restart and step == 2:
                path = str(tmp_path / "t.npz")
                g.write_solution(path)
                g.close()
                g = Solver(m, c)
                g.read_solution(path)
            g.run_time_step(3, tol=0.0)
        runs.append({k: g.get(k) for k in STATE + ("old", "oldold")})
        runs[-1]["t"] = g.time_state()
        g.close()
    for k in STATE + ("old", "oldold"):
        assert np.array_equal(runs[0][k], runs[1][k]), k
    assert runs[0]["t"] == runs[1]["t"]


# ------------------------------------------------- adaptive time step
def test_oracle_adaptive_time_step_at_rest():
    """AdaptiveTimeStep on a uniform n^3 cavity at rest (mdot = 0): a corner
    cell has three interior faces (mu h each) and three no-slip wall faces
    (mu h^2 / (h/2) each), the largest diffusion sum, 9 mu h; so dtlocal =
    Courant rho h^2 / (9 mu), then the change-factor clamp."""
    import oracle
    n = 6
    m, c = cs.cavity(n, jitter=0.0, unsteady=True, transient_scheme="euler", dt=0.05)
    o = oracle.Oracle(m, c)
    h = 1.0 / n
    want = 2.0 * c.rho * h * h / (9.0 * c.mu)
    got = o.adaptive_time_step(2.0, 1e-6, 1e6)
    assert abs(got - want) <= 1e-13 * want
    # clamps against the current dt (0.05): [0.5 dt, 5 dt]
    assert o.adaptive_time_step(2.0, 0.5, 5.0) == pytest.approx(min(max(want, 0.025), 0.25), rel=1e-13)
    assert o.adaptive_time_step(1e-9, 0.5, 5.0) == 0.025
    assert o.adaptive_time_step(1e9, 0.5, 5.0) == 0.25


def _adaptive_case(which):
    kw = dict(unsteady=True, transient_scheme="euler", dt=0.05, solver_mom="bicgs", solver_cont="bicgs",
              krylov_tol=1e-13, krylov_maxit=400)
    if which == "cavity3d":
        return cs.cavity(8, nz=6, jitter=0.2, seed=0, **kw)
    if which == "cavity2d":   # z patches are symmetry planes
        return cs.cavity(10, nz=1, jitter=0.2, seed=1, **kw)
    return cs.bfs(24, 9, 6, re_h=100.0, turbulence=False, **kw)   # velocity inlet, fully developed outlet


@pytest.mark.gpu
@pytest.mark.parametrize("which", ["cavity3d", "cavity2d", "step"])
def test_adaptive_time_step_matches_oracle(which):
    """fs_adaptive_time_step against the restatement on the same state (the
    oracle's mass fluxes copied into the device context): the unclamped
    dtlocal and the clamped dt agree to 1e-13 relative, over two time steps
    of no-slip walls, symmetry planes and a velocity inlet with outflow."""
    import oracle
    from flowsolversourcecode_b200.solver import Solver
    m, c = _adaptive_case(which)
    o = oracle.Oracle(m, c)
    g = Solver(m, c)
    if which == "step":
        for k, v in cs.bfs_initial_state(m, c, seed=0).items():
            o.set(k, v)
            g.set(k, v)
        o.initialize_mdot()
        g.initialize_mdot()
    else:
        _seed(o, o.N, 3)
        _seed(g, o.N, 3)
    for step in range(2):
        o.simple_iteration()
        g.simple_iteration()
        for k in ("mdot", "bmdot"):
            g.set(k, o.get(k))
        free_o = o.adaptive_time_step(2.0, 1e-9, 1e9)
        free_g = g.adaptive_time_step(2.0, 1e-9, 1e9)
        assert free_o > 0.0
        assert abs(free_g - free_o) <= 1e-13 * free_o, (step, free_g, free_o)
        dt_o = o.adaptive_time_step()
        dt_g = g.adaptive_time_step()
        assert abs(dt_g - dt_o) <= 1e-13 * dt_o, (step, dt_g, dt_o)
        o.advance_time(dt_o)
        g.advance_time(dt_o)
    assert g.time_state()["dt"] == o.get_time()["dt"]
    g.close()


@pytest.mark.gpu
def test_adaptive_time_step_rejects_unbuilt_forms():
    """Turbulent (and energy) cases have k, epsilon and temperature limits
    the device path does not build: the call fails with FS_E_ARG."""
    from flowsolversourcecode_b200.solver import Solver
    m, c = cs.bfs(24, 9, 6, turbulence=True, unsteady=True, transient_scheme="euler", dt=0.05)
    g = Solver(m, c)
    with pytest.raises(Exception):
        g.adaptive_time_step()
    g.close()
