"""GPU (sm_100a) path vs the CPU restatement, through the C ABI.

Tolerances: the per-face/per-cell kernels keep the reference's operation and
summation order (cell gathers visit faces in face order, --fmad=false), so
geometry, gradients, assembled coefficients, Rhie-Chow fluxes and the
corrections are compared at 1e-14 relative (they are expected to be
bit-identical; the test reports how many entries differ at all).  Krylov
solves differ only through the order of the FP64 dot-product sums (1e-9).
Converged fields are compared at 1e-8 relative L2.
"""
import numpy as np
import pytest

from flowsolversourcecode_b200 import case as cs

pytestmark = pytest.mark.gpu


def _pair(mesh, case):
    import oracle
    from flowsolversourcecode_b200.solver import Solver
    return Solver(mesh, case), oracle.Oracle(mesh, case)


def _rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    scale = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / scale)


def _close(name, gpu, ref, tol=1e-14):
    r = _rel(gpu, ref)
    ndiff = int(np.count_nonzero(np.asarray(gpu) != np.asarray(ref)))
    assert r <= tol, f"{name}: rel {r:.3e} ({ndiff} of {np.size(ref)} entries differ)"
    return ndiff


def _blocks(a, n):
    return [a[k * n:(k + 1) * n] for k in range(3)]


@pytest.fixture(scope="module")
def distorted():
    return cs.cavity(10, nz=8, jitter=0.2, seed=0, conv_scheme="sou", niter_start_hr=1)


def test_geometry(distorted):
    mesh, case = distorted
    s, o = _pair(mesh, case)
    _close("vol", s.get("volume"), o.get("vol"))
    xc = _blocks(s.get("xc"), s.N)
    for k, c in enumerate("xyz"):
        _close("xc" + c, xc[k], o.get(c + "c"))
    _close("gf", s.get("gfactor"), o.get("gf"))
    _close("gdiff", s.get("gdiff"), o.get("gdiff"))
    sf, ft, bsf = _blocks(s.get("sf"), s.F), _blocks(s.get("ft"), s.F), _blocks(s.get("bsf"), s.B)
    for k, c in enumerate("xyz"):
        _close("S" + c, sf[k], o.get("s" + c))
        _close("T" + c, ft[k], o.get("T" + c))
        _close("bS" + c, bsf[k], o.get("bs" + c))


def test_connectivity(distorted):
    mesh, case = distorted
    s, o = _pair(mesh, case)
    c = s.connectivity()
    assert np.array_equal(c["ncf"], o.get("ncf"))
    assert np.array_equal(c["cf"], o.get("cf"))
    assert np.array_equal(c["cn"], o.get("cn"))
    assert np.array_equal(c["own_slot"], o.get("own_slot"))
    assert np.array_equal(c["nbr_slot"], o.get("nbr_slot"))


@pytest.mark.parametrize("var,method", [("press", 2), ("press", 1), ("velx", 2), ("pressc", 2)])
def test_gradient(distorted, var, method):
    mesh, case = distorted
    s, o = _pair(mesh, case)
    rng = np.random.default_rng(1)
    phi = rng.standard_normal(s.N)
    bphi = rng.standard_normal(s.B)
    from flowsolversourcecode_b200 import _lib as L
    vid = {"velx": L.VAR_U, "pressc": L.VAR_PC, "press": L.VAR_P}[var]
    g, bg = s.gradient_host(var, method, 2, phi, bphi)
    go, bgo = o.gradient(vid, method, 2, phi, bphi)
    _close("grad", g, go)
    _close("bgrad", bg, bgo)


def _random_state(s, o, seed=0, scale=0.1):
    rng = np.random.default_rng(seed)
    N = s.N
    st = {}
    for k in ("u", "v", "w", "p"):
        st[k] = scale * rng.standard_normal(N)
    # a face flux consistent in magnitude with the velocities
    st["mdot"] = scale * 0.01 * rng.standard_normal(s.F)
    for k, v in st.items():
        s.set(k, v)
        o.set(k, v)
    return st


def test_momentum_assembly(distorted):
    mesh, case = distorted
    s, o = _pair(mesh, case)
    _random_state(s, o)
    s.set_iteration(3); o.set_iter(3)
    for comp in range(3):
        if comp > 0:   # the reference solves X before assembling Y: perturb the solved field
            name = "uvw"[comp - 1]
            val = s.get(name) * 1.01 + 1e-3
            s.set(name, val); o.set(name, val)
        s.assemble_momentum(comp)
        o.assemble_momentum(comp)
        _close(f"ac{comp}", s.get("ac"), o.get("ac"))
        _close(f"anb{comp}", s.get("anb"), o.get("anb"))
        _close(f"bc{comp}", s.get("bc"), o.get("bc"))
        d1 = ("du1", "dv1", "dw1")[comp]
        d2 = ("du2", "dv2", "dw2")[comp]
        _close(d1, s.get(d1), o.get(d1))
        _close(d2, s.get(d2), o.get(d2))
    for g in ("ugrad", "vgrad", "wgrad", "pgrad"):
        _close(g, s.get(g), o.get(g[0] + "g"))


def test_continuity_assembly_and_correction(distorted):
    mesh, case = distorted
    s, o = _pair(mesh, case)
    _random_state(s, o, seed=2)
    s.set_iteration(2); o.set_iter(2)
    for comp in range(3):
        s.assemble_momentum(comp); o.assemble_momentum(comp)
    s.assemble_continuity(); o.assemble_continuity()
    _close("mdot", s.get("mdot"), o.get("mdot"))
    _close("ac_p", s.get("ac"), o.get("ac"))
    _close("anb_p", s.get("anb"), o.get("anb"))
    _close("bc_p", s.get("bc"), o.get("bc"))
    pc = np.random.default_rng(5).standard_normal(s.N) * 1e-3
    s.set("pc", pc); o.set("pc", pc)
    s.correct_continuity(); o.correct_continuity()
    for k in ("u", "v", "w", "p", "mdot", "bp", "bu", "bv", "bw"):
        _close(k, s.get(k), o.get(k))
    _close("pcgrad", s.get("pcgrad"), o.get("pcg"))
    s.PrintConvergenceHistory()
    r = s.residuals
    ro = o.residuals()
    assert abs(r["max"][4] - ro["max"][4]) <= 1e-14 * ro["max"][4]
    assert abs(r["abs"][4] - ro["abs"][4]) <= 1e-12 * ro["abs"][4]


def test_bicgstab_parity():
    mesh, case = cs.cavity(12, nz=10, jitter=0.2, seed=3)
    s, o = _pair(mesh, case)
    for _ in range(3):
        o.simple_iteration()
    o.assemble_continuity()
    ac, anb, bc = o.get("ac"), o.get("anb"), o.get("bc")
    o.arr("kx")[:] = 0.0   # BICGSTAB_OMP's persistent x: start both from zero
    it_o = o.bicgstab(100, 1e-5)
    x_o = o.get("dphi")
    x_g, it_g = s.solve_system(ac, anb, bc, solver="bicgs")
    assert abs(it_g - it_o) <= 1, (it_g, it_o)
    assert _rel(x_g, x_o) <= 1e-6


def test_gmres_parity():
    # GMRES_RESTARTED_OMP_RETURNR on a momentum system (non-symmetric: SOU
    # convection) and on the p' system; the GPU's dot products sum in another
    # order, so both reach the 1e-9 normalised residual along slightly
    # different paths
    mesh, case = cs.cavity(12, nz=10, jitter=0.2, seed=3, conv_scheme="sou", niter_start_hr=1)
    s, o = _pair(mesh, case)
    for _ in range(3):
        o.simple_iteration()
    o.set_iter(4)
    for assemble in (lambda: o.assemble_momentum(0), o.assemble_continuity):
        assemble()
        ac, anb, bc = o.get("ac"), o.get("anb"), o.get("bc")
        it_o = o.gmres()
        x_o = o.get("dphi")
        x_g, it_g = s.solve_system(ac, anb, bc, solver="gmres")
        assert it_g > 0 and abs(it_g - it_o) <= max(5, it_o // 5), (it_g, it_o)
        assert _rel(x_g, x_o) <= 1e-6


def test_outer_iterations_gmres():
    # p' by GMRES through SolveEquation for three SIMPLE iterations; momentum by
    # BiCGSTAB to 1e-10 from a non-zero state, as in test_outer_iterations_bicgs
    # (multicolour SOR at rrF 0.01 would differ from the sequential sweep)
    mesh, case = cs.cavity(10, nz=8, jitter=0.2, seed=2, solver_mom="bicgs", solver_cont="gmres",
                           krylov_tol=1e-10, krylov_maxit=400)
    s, o = _pair(mesh, case)
    _random_state(s, o, seed=5, scale=0.05)
    for _ in range(3):
        s.simple_iteration()
        o.simple_iteration()
    for k in ("u", "v", "w", "p"):
        assert _rel(s.get(k), o.get(k)) <= 1e-6, k


def test_sor_solution():
    mesh, case = cs.cavity(12, nz=10, jitter=0.2, seed=3)
    s, o = _pair(mesh, case)
    for _ in range(2):
        o.simple_iteration()
    o.set_iter(3)
    o.assemble_momentum(0)
    ac, anb, bc = o.get("ac"), o.get("anb"), o.get("bc")
    x_g, it = s.solve_system(ac, anb, bc, rrf=1e-12, itmax=2000, solver="sor")
    fi = np.zeros(o.N)
    o.lib.om_solve_equation(o.h, 1, fi.ctypes.data, 1e-12, 2000, 0)
    assert _rel(x_g, fi) <= 1e-9


def test_ilu_sweeps_bit_identical():
    """'ilu' (FactorizeUsingILU.for, ILUMethod.for): the level-scheduled GPU
    factorisation and sweeps apply every term in the element-order loops'
    order, so a fixed number of sweeps gives the restatement's dphi bit for
    bit (rrF 0: no early stop, whose sum|r| test sums in another order)."""
    mesh, case = cs.cavity(12, nz=10, jitter=0.2, seed=3)
    s, o = _pair(mesh, case)
    for _ in range(2):
        o.simple_iteration()
    o.set_iter(3)
    for assemble in (lambda: o.assemble_momentum(0), o.assemble_continuity):
        assemble()
        ac, anb, bc = o.get("ac"), o.get("anb"), o.get("bc")
        x_g, it = s.solve_system(ac, anb, bc, rrf=0.0, itmax=7, solver="ilu")
        fi = np.zeros(o.N)
        o.lib.om_solve_equation(o.h, 1, fi.ctypes.data, 0.0, 7, 6)
        assert it == 7
        assert np.array_equal(x_g, fi)
    # to a tolerance: the converged solution
    x_g, it = s.solve_system(ac, anb, bc, rrf=1e-12, itmax=5000, solver="ilu")
    fi = np.zeros(o.N)
    o.lib.om_solve_equation(o.h, 1, fi.ctypes.data, 1e-12, 5000, 6)
    assert _rel(x_g, fi) <= 1e-9


def test_pbcg_matches_restatement():
    """'pbcg' (PBCGMethod.for): the same factorisation (bit for bit) and the
    same recurrence; only the order of the two dot products per iteration
    differs, so a fixed number of iterations agrees to rounding, and the
    iterations to rrF agree on the momentum and p' systems."""
    mesh, case = cs.cavity(12, nz=10, jitter=0.2, seed=3)
    s, o = _pair(mesh, case)
    for _ in range(2):
        o.simple_iteration()
    o.set_iter(3)
    for assemble in (lambda: o.assemble_momentum(0), o.assemble_continuity):
        assemble()
        ac, anb, bc = o.get("ac"), o.get("anb"), o.get("bc")
        x_g, it = s.solve_system(ac, anb, bc, rrf=0.0, itmax=6, solver="pbcg")
        fi = np.zeros(o.N)
        o.lib.om_solve_equation(o.h, 1, fi.ctypes.data, 0.0, 6, 8)
        assert it == 6
        assert _rel(x_g, fi) <= 1e-10
        x_g, it = s.solve_system(ac, anb, bc, rrf=0.05, itmax=200, solver="pbcg")
        fi = np.zeros(o.N)
        o.lib.om_solve_equation(o.h, 1, fi.ctypes.data, 0.05, 200, 8)
        assert it == o.lin_iters(1)
        assert _rel(x_g, fi) <= 1e-9


def test_outer_iterations_bicgs():
    # non-zero initial velocities so no momentum system has a zero right-hand side
    mesh, case = cs.cavity(10, nz=8, jitter=0.2, seed=1, conv_scheme="sou", niter_start_hr=1,
                           solver_mom="bicgs", solver_cont="bicgs", krylov_tol=1e-10, krylov_maxit=400)
    s, o = _pair(mesh, case)
    _random_state(s, o, seed=7, scale=0.05)
    for it in range(4):
        r = s.simple_iteration()
        o.simple_iteration()
        ro = o.residuals()
        for q in (0, 1, 2, 4):
            # residuals at round-off level (the 1e-10 Krylov solves leave ~1e-17
            # mass imbalance) are compared against an absolute floor
            floor = 1e-12 * max(ro["max"][0], ro["max"][1], ro["max"][2])
            assert abs(r["max"][q] - ro["max"][q]) <= max(1e-6 * ro["max"][q], floor), (it, q)
    for k in ("u", "v", "w", "p", "mdot"):
        assert _rel(s.get(k), o.get(k)) <= 1e-7, k


def test_converged_cavity2d():
    mesh, case = cs.cavity(24, nz=1, nstop_type=3)
    s, o = _pair(mesh, case)
    for _ in range(400):
        r = s.simple_iteration()
        o.simple_iteration()
    assert r["source"] < 1e-12
    for k in ("u", "v", "p"):
        a, b = s.get(k), o.get(k)
        if k == "p":
            a, b = a - a[0], b - b[0]
        assert np.linalg.norm(a - b) <= 1e-8 * np.linalg.norm(b), k


def test_deterministic():
    mesh, case = cs.cavity(12, nz=12, conv_scheme="sou", niter_start_hr=1)
    from flowsolversourcecode_b200.solver import Solver
    outs = []
    for _ in range(2):
        s = Solver(mesh, case)
        for _ in range(3):
            s.simple_iteration()
        outs.append({k: s.get(k) for k in ("u", "v", "w", "p", "mdot")})
        s.close()
    for k in outs[0]:
        assert np.array_equal(outs[0][k], outs[1][k]), k


def test_host_buffers_iteration():
    mesh, case = cs.cavity(10, nz=10)
    from flowsolversourcecode_b200.solver import Solver
    a, b = Solver(mesh, case), Solver(mesh, case)
    st = b.state()
    for _ in range(2):
        a.simple_iteration()
        b.simple_iteration_host(st)
    for k in st:
        assert np.array_equal(a.get(k), st[k]), k


def test_multigrid_parent_maps():
    mesh, case = cs.cavity(14, nz=12, jitter=0.2, seed=2, solver_cont="amg")
    import ctypes as C
    s, o = _pair(mesh, case)
    L = o.mg_setup()
    n = C.c_int32()
    sizes = np.zeros(16, np.int32)
    from flowsolversourcecode_b200 import _lib as Lb
    assert s.lib.fs_mg_levels(s.ctx, C.byref(n), Lb.iptr(sizes), 16) == 0
    assert n.value == L
    for l in range(L - 1):
        po = o.mg_parents(l)
        pg = np.zeros(po.shape[0], np.int32)
        assert s.lib.fs_mg_parents(s.ctx, l, Lb.iptr(pg), pg.shape[0]) == 0
        assert np.array_equal(pg, po), l


def _scipy_solution(o):
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla
    N, W = o.N, o.W
    ac, anb, cn = o.get("ac"), o.get("anb").reshape(W, N), o.get("cn").reshape(W, N)
    rows, cols, vals = list(range(N)), list(range(N)), list(ac)
    for j in range(W):
        m = cn[j] >= 0
        rows += list(np.nonzero(m)[0]); cols += list(cn[j][m]); vals += list(anb[j][m])
    A = sp.csr_matrix((vals, (rows, cols)), shape=(N, N))
    return A, spla.spsolve(A.tocsc(), o.get("bc"))


@pytest.mark.parametrize("solver,tol", [("amg", 1e-6), ("amg_bicgs", 1e-8), ("amg32_bicgs", 1e-8),
                                        ("amg32gs_bicgs", 1e-8)])
def test_multigrid_solvers_momentum_system(solver, tol):
    mesh, case = cs.cavity(16, nz=14, jitter=0.2, seed=3, krylov_tol=1e-10, krylov_maxit=200,
                           mg_max_cycles=200)
    s, o = _pair(mesh, case)
    for _ in range(2):
        o.simple_iteration()
    o.set_iter(3)
    o.assemble_momentum(0)
    A, x_direct = _scipy_solution(o)
    x, it = s.solve_system(o.get("ac"), o.get("anb"), o.get("bc"), rrf=1e-10, itmax=200, solver=solver)
    assert it >= 1
    assert _rel(x, x_direct) <= tol, (solver, it, _rel(x, x_direct))


@pytest.mark.parametrize("solver", ["amg_bicgs", "amg32_bicgs", "amg32gs_bicgs", "amg"])
def test_multigrid_pressure_correction_residual(solver):
    # the closed-cavity p' system is singular: check the residual, and the
    # solution up to the constant null vector
    mesh, case = cs.cavity(16, nz=14, jitter=0.2, seed=3, krylov_tol=1e-9, krylov_maxit=200, mg_max_cycles=200)
    s, o = _pair(mesh, case)
    for _ in range(3):
        o.simple_iteration()
    o.assemble_continuity()
    A, _ = _scipy_solution(o)
    b = o.get("bc")
    x, it = s.solve_system(o.get("ac"), o.get("anb"), b, rrf=1e-9, itmax=200, solver=solver)
    res = np.linalg.norm(b - A @ x) / np.linalg.norm(b)
    assert res <= (1e-8 if solver != "amg" else 1e-6), (solver, it, res)


def test_simple_iterations_with_amg_bicgs():
    mesh, case = cs.cavity3d(16, solver_cont="amg_bicgs", krylov_tol=1e-8)
    from flowsolversourcecode_b200.solver import Solver
    s = Solver(mesh, case)
    hist = [s.simple_iteration()["source"] for _ in range(30)]
    assert np.isfinite(hist).all()
    assert hist[-1] < hist[1]


def test_batched_momentum_same_fixed_point():
    # X, Y, Z solved together: the per-iteration wall cross terms lag, the
    # converged field is the same
    from flowsolversourcecode_b200.solver import Solver
    mesh, case = cs.cavity(12, nz=10, re=100.0, nstop_type=3)
    _, case_b = cs.cavity(12, nz=10, re=100.0, nstop_type=3, batched_momentum=True)
    a, b = Solver(mesh, case), Solver(mesh, case_b)
    for _ in range(400):
        ra = a.simple_iteration()
        rb = b.simple_iteration()
    assert ra["source"] < 1e-11 and rb["source"] < 1e-11
    for k in ("u", "v", "w"):
        x, y = a.get(k), b.get(k)
        assert np.linalg.norm(x - y) <= 1e-8 * np.linalg.norm(x), k


def test_three_component_finish_matches_per_component_assembly():
    # the multi-RHS form finishes u, v, w in one launch; from the same fields
    # the D values it leaves equal, bit for bit, those of the three separate
    # X/Y/Z assemblies
    from flowsolversourcecode_b200.solver import Solver
    mesh, case = cs.cavity(10, nz=8, jitter=0.2, seed=1, re=400.0, conv_scheme="sou", niter_start_hr=1,
                           batched_momentum=True)
    a, b = Solver(mesh, case), Solver(mesh, case)
    rng = np.random.default_rng(3)
    for k in ("u", "v", "w", "p"):
        x = 0.05 * rng.standard_normal(a.N)
        a.set(k, x)
        b.set(k, x)
    a.set_iteration(1)
    ref = {}
    for c, names in enumerate((("du1", "du2"), ("dv1", "dv2"), ("dw1", "dw2"))):
        a.assemble_momentum(c)
        for k in names:
            ref[k] = a.get(k)
    b.set_iteration(0)
    b.simple_iteration()
    for k, x in ref.items():
        assert np.array_equal(b.get(k), x), k
    a.close()
    b.close()


def test_bounded_wait_runs_out_and_reports_timeout():
    # Failure detection without a GPU fault: the AMG preconditioner's team
    # barriers are made to wait for one CTA more than takes part, so their
    # bounded polls run out; the iteration must come back with FS_E_TIMEOUT in
    # about a second, and the device and the library must stay usable.
    import ctypes as C
    import time
    from flowsolversourcecode_b200 import _lib as Lb
    from flowsolversourcecode_b200.solver import Solver
    mesh, case = cs.cavity(12, nz=12, solver_cont="amg_bicgs", krylov_tol=1e-8, krylov_maxit=50)
    s = Solver(mesh, case)
    s.simple_iteration()
    assert s.lib.fs_test_wait_timeout(s.ctx, 1) == 0
    r = Lb.FsResiduals()
    t0 = time.time()
    rc = s.lib.fs_simple_iteration(s.ctx, C.byref(r))
    dt = time.time() - t0
    assert rc == Lb.FS_E_TIMEOUT, rc
    assert dt < 10.0, dt
    assert b"timed out" in s.lib.fs_last_error(s.ctx)
    assert s.lib.fs_test_wait_timeout(s.ctx, 0) == 0
    s.close()
    t = Solver(mesh, case)
    for _ in range(2):
        res = t.simple_iteration()
    assert np.isfinite(res["source"])
    t.close()
