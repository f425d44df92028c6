"""CPU oracle of the learned p' initial-guess network -- TEST INFRASTRUCTURE ONLY.

The network has no reference counterpart (the reference starts every p' solve
from zero), so this restatement is pinned by finite differences of its own
loss (tests/test_nn_oracle.py), not by the reference.  It mirrors the GPU
kernels of flowsolversourcecode_b200/csrc/fs_nn.cu term by term:

  h0 = relu(X W_in + b_in)                                   X: N x 8
  layer l: m = sum_s wgt[s, i] h[cn[s, i]]  (slot order)      wgt, cn: W x N
           z = [h, m] W_l + b_l ;  h <- h + relu(z)            4 layers, width 64
  y = h w_out + b_out
  loss = sum((y - mean y) - t)^2 / sum t^2

With bf16=True the operands of the layer products are rounded to bfloat16
(round to nearest even) as the tensor-core kernels do, with FP32 activations
and FP64 sums standing in for FP32 accumulation; with bf16=False everything is
float64 (the mode the finite-difference check uses).  The aggregation is
symmetric (wgt[s_i(k), i] == wgt[s_k(i), k]), so its transpose is the same
gather -- the GPU backward relies on it and so does this one.
"""
from __future__ import annotations

import numpy as np

F_IN, H, K, L = 8, 64, 128, 4
OFF_WIN = 0
OFF_BIN = F_IN * H
def OFF_L(l): return OFF_BIN + H + l * (K * H + H)
OFF_WOUT = OFF_L(L)
OFF_BOUT = OFF_WOUT + H
NPARAM = OFF_BOUT + 1


def bf16_round(a) -> np.ndarray:
    """float32 -> bfloat16 -> float32, round to nearest even."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def unpack(theta: np.ndarray) -> dict:
    p = {"W_in": theta[OFF_WIN:OFF_WIN + F_IN * H].reshape(F_IN, H), "b_in": theta[OFF_BIN:OFF_BIN + H]}
    for l in range(L):
        o = OFF_L(l)
        p[f"W{l}"] = theta[o:o + K * H].reshape(K, H)
        p[f"b{l}"] = theta[o + K * H:o + K * H + H]
    p["w_out"] = theta[OFF_WOUT:OFF_WOUT + H]
    p["b_out"] = theta[OFF_BOUT]
    return p


def gather(wgt: np.ndarray, cn: np.ndarray, h: np.ndarray, dtype) -> np.ndarray:
    """m_i = sum over slots s of wgt[s, i] h[cn[s, i]] in slot order."""
    m = np.zeros_like(h, dtype=dtype)
    for s in range(cn.shape[0]):
        k = cn[s]
        ok = k >= 0
        contrib = np.zeros_like(h, dtype=dtype)
        contrib[ok] = (wgt[s, ok].astype(dtype)[:, None] * h[k[ok]].astype(dtype)).astype(dtype)
        m = (m + contrib).astype(dtype)
    return m


def forward(theta, X, wgt, cn, bf16: bool = True) -> dict:
    dt = np.float32 if bf16 else np.float64
    p = unpack(np.asarray(theta, dt))
    X = np.asarray(X, dt)
    z0 = (X.astype(np.float64) @ p["W_in"].astype(np.float64) + p["b_in"]).astype(dt)
    h = np.maximum(z0, 0).astype(dt)
    cache = {"X": X, "z0": z0, "h": [h], "m": [], "z": []}
    for l in range(L):
        m = gather(wgt, cn, h, dt)
        A = np.concatenate([h, m], axis=1)
        Wl = p[f"W{l}"]
        if bf16:
            A, Wl = bf16_round(A), bf16_round(Wl)
        z = (A.astype(np.float64) @ Wl.astype(np.float64) + p[f"b{l}"]).astype(dt)
        h = (h + np.maximum(z, 0)).astype(dt)
        cache["m"].append(m)
        cache["z"].append(z)
        cache["h"].append(h)
    y = (h.astype(np.float64) @ p["w_out"].astype(np.float64) + p["b_out"]).astype(dt)
    cache["y"] = y
    return cache


def loss_and_grad(theta, X, wgt, cn, t, bf16: bool = True):
    """Loss and gradient (flat, parameter order of the GPU vector)."""
    dt = np.float32 if bf16 else np.float64
    c = forward(theta, X, wgt, cn, bf16)
    p = unpack(np.asarray(theta, dt))
    t = np.asarray(t, np.float64)
    y = c["y"].astype(np.float64)
    tt = float(np.sum(t * t)) or 1.0
    d = (y - y.mean()) - t
    loss = float(np.sum(d * d) / tt)
    dy = (2.0 * d / tt).astype(dt)
    g = np.zeros(NPARAM, np.float64)
    h4 = c["h"][L].astype(np.float64)
    g[OFF_WOUT:OFF_WOUT + H] = h4.T @ dy.astype(np.float64)
    g[OFF_BOUT] = float(np.sum(dy, dtype=np.float64))
    dh = (dy[:, None].astype(np.float64) * p["w_out"].astype(np.float64)[None, :]).astype(dt)
    for l in range(L - 1, -1, -1):
        z = c["z"][l]
        dz = np.where(z > 0, dh, 0).astype(dt)
        A = np.concatenate([c["h"][l], c["m"][l]], axis=1)
        Wl = p[f"W{l}"]
        dzo = dz
        if bf16:
            A, Wl, dzo = bf16_round(A), bf16_round(Wl), bf16_round(dz)
        o = OFF_L(l)
        g[o:o + K * H] = (A.astype(np.float64).T @ dzo.astype(np.float64)).ravel()
        g[o + K * H:o + K * H + H] = dz.astype(np.float64).sum(axis=0)
        dA = (dzo.astype(np.float64) @ Wl.astype(np.float64).T).astype(dt)
        dh_new = (dh + dA[:, :H]).astype(dt)
        dh = (dh_new + gather(wgt, cn, dA[:, H:], dt)).astype(dt)
    dz0 = np.where(c["z0"] > 0, dh, 0).astype(np.float64)
    g[OFF_WIN:OFF_WIN + F_IN * H] = (c["X"].astype(np.float64).T @ dz0).ravel()
    g[OFF_BIN:OFF_BIN + H] = dz0.sum(axis=0)
    return loss, g, c["y"]


def symmetric_weights(cf: np.ndarray, cn: np.ndarray, face_w: np.ndarray) -> np.ndarray:
    """Slot weights wgt[s, i] = face_w[face of slot s] on interior slots, 0
    elsewhere: symmetric by construction, like the GPU's c_f / sqrt(ac_i ac_j)."""
    w = np.zeros(cn.shape, np.float32)
    ok = cn >= 0
    w[ok] = face_w[cf[ok]]
    return w
