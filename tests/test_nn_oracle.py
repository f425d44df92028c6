"""The CPU oracle of the learned-guess network, pinned by finite differences
(the network has no reference counterpart).  CPU only."""
import numpy as np
import pytest

from flowsolversourcecode_b200 import mesh as fm
from oracle import nn_oracle as nno


def graph(nx=4, ny=3, nz=3):
    """Slot-major neighbour and face tables of a box mesh (interior faces)."""
    m = fm.box_mesh(nx, ny, nz)
    N = m.n_cells
    slots = [[] for _ in range(N)]
    for f in range(m.n_internal):
        o, n = int(m.owner[f]), int(m.neighbour[f])
        slots[o].append((n, f))
        slots[n].append((o, f))
    W = max(len(s) for s in slots)
    cn = -np.ones((W, N), np.int32)
    cf = np.zeros((W, N), np.int32)
    for i, s in enumerate(slots):
        for j, (k, f) in enumerate(s):
            cn[j, i], cf[j, i] = k, f
    return m, cn, cf


def random_case(seed=0, nx=4, ny=3, nz=3):
    rng = np.random.default_rng(seed)
    m, cn, cf = graph(nx, ny, nz)
    N = cn.shape[1]
    X = rng.standard_normal((N, nno.F_IN)).astype(np.float32)
    X[:, 7] = 1.0
    wgt = nno.symmetric_weights(cf, cn, rng.uniform(0.05, 0.3, m.n_internal).astype(np.float32))
    theta = (0.2 * rng.standard_normal(nno.NPARAM)).astype(np.float32)
    t = rng.standard_normal(N)
    t -= t.mean()
    return theta, X, wgt, cn, t


def test_weights_symmetric():
    _, _, wgt, cn, _ = random_case()
    N = cn.shape[1]
    for i in range(N):
        for s in range(cn.shape[0]):
            k = cn[s, i]
            if k < 0:
                continue
            back = [q for q in range(cn.shape[0]) if cn[q, k] == i]
            assert len(back) == 1 and wgt[back[0], k] == wgt[s, i]


def test_gradient_matches_finite_differences():
    theta, X, wgt, cn, t = random_case(1)
    th = theta.astype(np.float64)
    loss, g, _ = nno.loss_and_grad(th, X, wgt, cn, t, bf16=False)
    rng = np.random.default_rng(7)
    # a sample of coordinates from every parameter block
    blocks = [(nno.OFF_WIN, nno.F_IN * nno.H), (nno.OFF_BIN, nno.H)]
    for l in range(nno.L):
        blocks += [(nno.OFF_L(l), nno.K * nno.H), (nno.OFF_L(l) + nno.K * nno.H, nno.H)]
    blocks += [(nno.OFF_WOUT, nno.H), (nno.OFF_BOUT, 1)]
    eps = 1e-6
    checked = 0
    for off, n in blocks:
        for q in rng.choice(n, size=min(4, n), replace=False):
            p = off + int(q)
            tp, tm = th.copy(), th.copy()
            tp[p] += eps
            tm[p] -= eps
            lp, _, _ = nno.loss_and_grad(tp, X, wgt, cn, t, bf16=False)
            lm, _, _ = nno.loss_and_grad(tm, X, wgt, cn, t, bf16=False)
            fd = (lp - lm) / (2 * eps)
            assert abs(fd - g[p]) <= 1e-5 * max(1.0, abs(fd)), (p, fd, g[p])
            checked += 1
    assert checked > 30 and loss > 0


def test_bf16_round_is_nearest_even():
    a = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -2.5, 0.0], np.float32)
    r = nno.bf16_round(a)
    assert r[0] == 1.0
    assert r[1] == 1.0                      # tie -> even mantissa
    assert r[2] == np.float32(1.0 + 2 ** -7)
    assert r[3] == -2.5 and r[4] == 0.0


def test_bf16_forward_close_to_fp64():
    theta, X, wgt, cn, t = random_case(2)
    y32 = nno.forward(theta, X, wgt, cn, bf16=True)["y"]
    y64 = nno.forward(theta.astype(np.float64), X, wgt, cn, bf16=False)["y"]
    assert np.linalg.norm(y32 - y64) / np.linalg.norm(y64) < 3e-2
