"""Failure detection of the SIMPLE loop, made on the host: a NaN planted in a
field must come back as FS_E_NAN, and a stop metric that grows by more than
FS_DIVERGENCE_FACTOR over its largest earlier value as FS_E_DIVERGED.  No
device fault is involved: every solver loop is bounded, so a NaN only ends
the Krylov and Gauss-Seidel loops early; the context stays usable."""
import numpy as np
import pytest

from flowsolversourcecode_b200 import case as cs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("solver_cont", ["bicgs", "amg_bicgs"])
def test_nan_in_a_field_reports_nan(solver_cont):
    from flowsolversourcecode_b200 import _lib as L
    from flowsolversourcecode_b200.solver import Solver
    mesh, case = cs.cavity(8, nz=6, solver_mom="sor", solver_cont=solver_cont, krylov_tol=1e-8,
                           krylov_maxit=100)
    s = Solver(mesh, case)
    for _ in range(2):
        s.simple_iteration()
    u = s.get("u")
    u[s.N // 2] = np.nan
    s.set("u", u)
    with pytest.raises(L.FsError) as e:
        s.simple_iteration()
    assert e.value.status == L.FS_E_NAN
    assert b"NaN" in s.lib.fs_last_error(s.ctx)
    s.close()
    t = Solver(mesh, case)                 # the device and the library stay usable
    r = t.simple_iteration()
    assert np.isfinite(r["source"])
    t.close()


def test_growing_residual_reports_divergence():
    from flowsolversourcecode_b200 import _lib as L
    from flowsolversourcecode_b200.solver import Solver
    mesh, case = cs.cavity(8, nz=6, solver_mom="sor", solver_cont="bicgs", krylov_tol=1e-8, krylov_maxit=100,
                           nstop_type=2)
    s = Solver(mesh, case)
    hist = [s.simple_iteration()["source"] for _ in range(3)]
    assert all(np.isfinite(hist))
    for k in ("u", "v", "w"):                  # a velocity 1e8 times too large
        s.set(k, 1e8 * s.get(k))
    with pytest.raises(L.FsError) as e:
        s.simple_iteration()
    assert e.value.status == L.FS_E_DIVERGED
    assert b"diverged" in s.lib.fs_last_error(s.ctx)
    s.close()


def test_converging_run_never_reports_divergence():
    from flowsolversourcecode_b200.solver import Solver
    mesh, case = cs.cavity(8, nz=1, solver_mom="sor", solver_cont="amg_bicgs", krylov_tol=1e-8,
                           krylov_maxit=100)
    s = Solver(mesh, case)
    hist = s.run(400, tol=1e-10)
    assert hist[-1]["source"] < 1e-10
    s.close()
