"""Learned p' initial guess on the GPU: the BF16 tensor-core forward/backward
kernels against the CPU oracle, training on snapshots the plain solver
captures, and what the trained guess gains over the zero start."""
import numpy as np
import pytest

from flowsolversourcecode_b200 import case as cs
from oracle import nn_oracle as nno

pytestmark = pytest.mark.gpu


def _solver(n=12, **kw):
    from flowsolversourcecode_b200.solver import Solver
    mesh, case = cs.cavity(n, re=100.0, **kw)
    return Solver(mesh, case)


@pytest.mark.parametrize("n", [12, 40])
def test_kernels_match_oracle(n):
    # 12^3: one 128-row tile per CTA of the persistent backward; 40^3 (500
    # tiles over 296 CTAs): CTAs that accumulate dW over two tiles in TMEM
    s = _solver(n)
    s.nn_create(0, seed=3)
    con = s.connectivity()
    W, N, F = s.W, s.N, s.F
    cn = con["cn"].reshape(W, N)
    cf = con["cf"].reshape(W, N)
    rng = np.random.default_rng(11)
    face_w = np.zeros(F, np.float32)
    face_w[:] = rng.uniform(0.05, 0.3, F)
    wgt = nno.symmetric_weights(cf, cn, face_w)
    X = rng.standard_normal((N, nno.F_IN)).astype(np.float32)
    X[:, 7] = 1.0
    theta = (0.15 * rng.standard_normal(nno.NPARAM)).astype(np.float32)
    t = rng.standard_normal(N)
    t -= t.mean()
    s.nn_params(set=theta)
    assert np.array_equal(s.nn_params(), theta)
    g = s.nn_eval(X, wgt.ravel(), t.astype(np.float32))
    loss, grad, y = nno.loss_and_grad(theta, X, wgt, cn, t.astype(np.float32), bf16=True)
    # FP32 accumulation order of the tensor-core products differs from the
    # oracle's FP64 sums; a rare bf16 rounding flip propagates a little
    assert np.linalg.norm(g["y"] - y) / np.linalg.norm(y) < 2e-3
    assert abs(g["loss"] - loss) / loss < 2e-3
    blocks = {"W_in": (nno.OFF_WIN, nno.F_IN * nno.H), "b_in": (nno.OFF_BIN, nno.H),
              "w_out": (nno.OFF_WOUT, nno.H + 1)}
    for l in range(nno.L):
        blocks[f"W{l}"] = (nno.OFF_L(l), nno.K * nno.H)
        blocks[f"b{l}"] = (nno.OFF_L(l) + nno.K * nno.H, nno.H)
    for name, (o, n) in blocks.items():
        a, b = g["grad"][o:o + n].astype(np.float64), grad[o:o + n]
        assert np.linalg.norm(a - b) <= 1e-2 * np.linalg.norm(b) + 1e-7, (name, np.linalg.norm(a - b), np.linalg.norm(b))
    s.close()


def _run(s, iters):
    its = []
    for _ in range(iters):
        r = s.simple_iteration()
        its.append(r["lin_iters"][3])
    return its


@pytest.mark.parametrize("solver", ["amg_bicgs", "amg32_bicgs"])
def test_training_and_gain(solver):
    n, warm, K = 16, 8, 40
    kw = dict(solver_cont=solver, krylov_tol=1e-8, krylov_maxit=200)
    # snapshots from the plain solver
    a = _solver(n, **kw)
    a.nn_create(snapshot_capacity=64, seed=5)
    a.nn_mode(capture=True, use=False)
    _run(a, 64)
    assert a.nn_snapshots() == 63          # the first solve has no previous p'
    first, last = a.nn_train(epochs=40, lr=2e-3, seed=1)
    assert np.isfinite(last) and last < 0.5 * first, (first, last)
    theta = a.nn_params()
    a.close()
    # same case from the start, with and without the trained guess
    b = _solver(n, **kw)
    c = _solver(n, **kw)
    c.nn_create(0, seed=5)
    c.nn_params(set=theta)
    c.nn_mode(capture=False, use=True)
    _run(b, warm)
    _run(c, warm)
    ib, ic = _run(b, K), _run(c, K)
    st = c.nn_stats()
    # the guess was tried; zero-start probes and parking take the other solves
    assert 0 < st["uses"] < warm + K
    for k in ("u", "v", "w", "p"):
        x, ref = c.get(k), b.get(k)
        assert np.linalg.norm(x - ref) <= 1e-6 * np.linalg.norm(ref), k
    # the guess never costs iterations beyond round-off (a bad guess falls back
    # to the zero start); report the gain
    print(f"\n{solver}: p' iterations over {K} outer iterations: zero start {sum(ib)}, "
          f"learned guess {sum(ic)}; policy {st}")
    assert sum(ic) <= sum(ib) + K // 10
    b.close()
    c.close()
