"""Ensemble case generation and sharding (CPU) and the graph-captured
ensemble run against ordinary per-case iterations (GPU)."""
import numpy as np
import pytest

from flowsolversourcecode_b200 import ensemble as E


def test_specs_seeded_and_in_range():
    a, b = E.make_specs(64, seed=0), E.make_specs(64, seed=0)
    assert a == b
    assert E.make_specs(64, seed=1) != a
    e = np.array([s.edge for s in a])
    assert e.min() >= 32 and e.max() <= 96
    assert all(0.5 <= s.lid <= 2.0 for s in a)
    assert all(100.0 <= s.re <= 2000.0 for s in a)
    # E[e^3] for e ~ U{32..96} is 327,680 cells per case
    assert 0.8 * 327680 * 64 < sum(s.cells for s in a) < 1.2 * 327680 * 64


def test_shard_covers_and_balances():
    sp = E.make_specs(64, seed=0)
    sizes = [s.cells for s in sp]
    for world in (1, 2, 4, 8):
        parts = E.shard(sizes, world)
        flat = sorted(q for p in parts for q in p)
        assert flat == list(range(64))
        loads = [sum(sizes[q] for q in p) for p in parts]
        assert max(loads) - min(loads) <= max(sizes)


@pytest.mark.gpu
def test_graph_run_matches_ordinary_iterations():
    from flowsolversourcecode_b200.solver import Solver
    specs = [E.CaseSpec(10, 1.0, 400.0), E.CaseSpec(12, 0.7, 150.0), E.CaseSpec(14, 1.6, 900.0)]
    cases = [E.build_case(s) for s in specs]
    ens = E.Ensemble(cases)
    out = ens.run(iters=3, launches=2)
    ens.close()
    for q, (m, c) in enumerate(cases):
        s = Solver(m, c)
        # the run starts after ordinary iterations that pass the HR start and fill the p' history
        warm = max(1, c.niter_start_hr, c.pc_history)
        ref = [s.simple_iteration()["source"] for _ in range(warm + 6)][warm:]
        s.close()
        assert np.allclose(out["source"][q], ref, rtol=1e-12, atol=0), (q, out["source"][q], ref)
    assert out["ms"] > 0 and out["cell_iters_per_s"] > 0


@pytest.mark.gpu
def test_autotune_picks_a_shape():
    specs = [E.CaseSpec(12, 1.0, 300.0), E.CaseSpec(16, 1.0, 300.0)]
    ens = E.Ensemble([E.build_case(s) for s in specs])
    shapes = ens.autotune(shapes=(1, 2, 4), iters=1)
    assert all(k in (1, 2, 4) for k in shapes)
    out = ens.run(iters=2, launches=1)
    assert np.all(np.isfinite(out["source"]))
    ens.close()


@pytest.mark.gpu
def test_batched_run_matches_sequential_within_tolerance():
    """The p' solves of all cases in one launch, a CTA group per case: the
    Krylov sums run over the group instead of the whole grid, so the results
    match the sequential graph run within the p' tolerance, not bit for bit."""
    specs = [E.CaseSpec(10, 1.0, 400.0), E.CaseSpec(12, 0.7, 150.0), E.CaseSpec(16, 1.6, 900.0)]
    outs = []
    for batched in (False, True):
        ens = E.Ensemble([E.build_case(s, krylov_tol=1e-10) for s in specs])
        outs.append(ens.run(iters=3, launches=2, batched=batched))
        ens.close()
    seq, bat = outs
    assert np.all(np.isfinite(bat["source"]))
    assert np.allclose(bat["source"], seq["source"], rtol=1e-6, atol=0), (bat["source"], seq["source"])
    assert np.all(np.abs(bat["pc_iters"] - seq["pc_iters"]) <= 2), (bat["pc_iters"], seq["pc_iters"])
    assert bat["ms"] > 0


@pytest.mark.gpu
def test_batched_run_rejects_mixed_solvers():
    from flowsolversourcecode_b200._lib import FsError
    a = E.build_case(E.CaseSpec(10, 1.0, 400.0))
    m, c = E.build_case(E.CaseSpec(12, 1.0, 400.0))
    c.solver_cont = "bicgs"
    ens = E.Ensemble([a, (m, c)])
    with pytest.raises(FsError):
        ens.run(iters=1, launches=1, batched=True)
    ens.close()


@pytest.mark.gpu
def test_split_autotune_picks_a_candidate():
    specs = [E.CaseSpec(10, 1.0, 400.0), E.CaseSpec(16, 1.0, 300.0)]
    ens = E.Ensemble([E.build_case(s) for s in specs])
    e = ens.autotune_split(exponents=(0.5, 1.0), iters=1)
    assert e in (0.5, 1.0) and set(ens.split_ms) == {0.5, 1.0}
    out = ens.run(iters=2, launches=1, batched=True)
    assert np.all(np.isfinite(out["source"]))
    ens.close()


def test_split_exponent_rejects_out_of_range():
    from flowsolversourcecode_b200 import _lib as L
    lib = L.load()
    assert lib.fs_ensemble_split(None, 1.0) == L.FS_E_ARG
