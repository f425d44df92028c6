"""writeSolution / readSolution: a run restarted from a written state repeats
the outer iterations of the run that wrote it, bit for bit."""
import os

import numpy as np
import pytest

from flowsolversourcecode_b200 import case as cs

pytestmark = pytest.mark.gpu


def _continue(make, setup, k, m, path):
    from flowsolversourcecode_b200.solver import Solver
    mesh, case = make()
    a = Solver(mesh, case)
    setup(a, mesh, case)
    for _ in range(k):
        a.simple_iteration()
    a.write_solution(path)
    ra = [a.simple_iteration()["source"] for _ in range(m)]
    fa = {f: a.get(f) for f in a.RESTART_FIELDS + (a.RESTART_TURB if case.turbulence else ())}
    a.close()
    b = Solver(mesh, case)
    b.read_solution(path)
    rb = [b.simple_iteration()["source"] for _ in range(m)]
    fb = {f: b.get(f) for f in fa}
    b.close()
    assert ra == rb
    for f in fa:
        assert np.array_equal(fa[f], fb[f]), f


def _none(s, mesh, case):
    pass


def _bfs_init(s, mesh, case):
    for k, v in cs.bfs_initial_state(mesh, case).items():
        s.set(k, v)
    s.initialize_mdot()


@pytest.mark.parametrize("solver", ["bicgs", "amg_bicgs"])
def test_restart_cavity(tmp_path, solver):
    make = lambda: cs.cavity3d(12, solver_cont=solver, krylov_tol=1e-8, krylov_maxit=200)
    _continue(make, _none, 4, 3, os.path.join(tmp_path, "cavity.npz"))


def test_restart_kepsilon_step(tmp_path):
    make = lambda: cs.bfs(24, 9, 6, solver_cont="amg_bicgs", krylov_tol=1e-8, krylov_maxit=200)
    _continue(make, _bfs_init, 3, 3, os.path.join(tmp_path, "step.npz"))
