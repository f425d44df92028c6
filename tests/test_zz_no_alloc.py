"""fs_bicgstab_noalloc: the BiCGSTAB solve for callers that cannot allocate
device memory (their device memory belongs to another allocator, or they may
not allocate once running).  It must give the same answer as the allocating
entry point fs_solve_system_host, on consecutive calls that share the
library's fixed scratch array.  Device buffers for the test itself come from
torch (the test is not such a caller)."""
import ctypes as C

import numpy as np
import pytest

from flowsolversourcecode_b200 import case as cs

pytestmark = pytest.mark.gpu


def _systems():
    import oracle
    mesh, case = cs.cavity(12, nz=10, jitter=0.2, seed=3)
    o = oracle.Oracle(mesh, case)
    for _ in range(2):
        o.simple_iteration()
    o.set_iter(3)
    o.assemble_continuity()             # p' system (singular, closed cavity)
    sys_a = (o.get("ac"), o.get("anb"), o.get("bc"))
    o.assemble_momentum(0)              # x-momentum system
    sys_b = (o.get("ac"), o.get("anb"), o.get("bc"))
    return mesh, case, o, [sys_a, sys_b]


def test_noalloc_matches_allocating_entry_point():
    import torch
    from flowsolversourcecode_b200 import _lib as L
    from flowsolversourcecode_b200.solver import Solver
    mesh, case, o, systems = _systems()
    lib = L.load()
    N, W = o.N, o.W
    dev = torch.device("cuda:0")
    ncf = torch.tensor(o.get("ncf"), dtype=torch.int32, device=dev)
    cn = torch.tensor(o.get("cn"), dtype=torch.int32, device=dev)
    iters = torch.zeros(1, dtype=torch.int32, device=dev)
    for k, (ac, anb, bc) in enumerate(systems):       # two calls in a row
        ref = Solver(mesh, case)                       # fresh context: its Krylov x starts at 0
        x_ref, it_ref = ref.solve_system(ac, anb, bc, solver="bicgs")
        ref.close()
        d_ac = torch.tensor(ac, device=dev)
        d_anb = torch.tensor(anb, device=dev)
        d_bc = torch.tensor(bc, device=dev)
        d_x = torch.zeros(N, dtype=torch.float64, device=dev)
        torch.cuda.synchronize()
        rc = lib.fs_bicgstab_noalloc(N, W, ncf.data_ptr(), cn.data_ptr(), d_ac.data_ptr(), d_anb.data_ptr(),
                                     d_bc.data_ptr(), d_x.data_ptr(), case.krylov_maxit, case.krylov_tol,
                                     iters.data_ptr(), None)
        assert rc == L.FS_OK
        torch.cuda.synchronize()
        x = d_x.cpu().numpy()
        assert int(iters.item()) == it_ref, (k, int(iters.item()), it_ref)
        scale = np.abs(x_ref).max()
        assert np.abs(x - x_ref).max() <= 1e-12 * scale, k


def test_noalloc_rejects_oversized_system():
    from flowsolversourcecode_b200 import _lib as L
    lib = L.load()
    n = L.FS_NOALLOC_MAX_ROWS + 1
    rc = lib.fs_bicgstab_noalloc(n, 6, 1, 1, 1, 1, 1, 1, 100, 1e-5, None, None)
    assert rc == L.FS_E_TOO_LARGE
