"""Test infrastructure: float64 numpy restatement of the learned
preconditioner's network (asgard_b200/csrc/mlp.cu) -- forward pass, MSE loss
and backward pass -- used to check the GPU kernels' gradients.  The network
has no counterpart in the reference; this file is the checker for the
project's own forward/backward kernels, not a product path.

Network (width H, GELU gates from the level features lam):
    g_l = gelu(lam P_l + p_l)          l = 1, 2, 3
    h_1 = g_1 * (u W_1),  h_l = g_l * (h_{l-1} W_l),  y = h_3 W_4
Flat parameter layout (asgk_mlp_get_params): W1 (ts x H), W2 (H x H),
W3 (H x H), W4 (H x ts), then P_l (d x H), p_l (H) for l = 1, 2, 3.
"""
from __future__ import annotations

import math

import numpy as np

_erf = np.vectorize(math.erf, otypes=[np.float64])


def gelu(x):
    return 0.5 * x * (1.0 + _erf(x / math.sqrt(2.0)))


def dgelu(x):
    cdf = 0.5 * (1.0 + _erf(x / math.sqrt(2.0)))
    pdf = np.exp(-0.5 * x * x) / math.sqrt(2.0 * math.pi)
    return cdf + x * pdf


def layout(ts, d, H):
    """(name, shape) of every parameter tensor in flat order."""
    return ([("W1", (ts, H)), ("W2", (H, H)), ("W3", (H, H)), ("W4", (H, ts))] +
            [item for l in (1, 2, 3) for item in ((f"P{l}", (d, H)), (f"p{l}", (H,)))])


def unpack(params, ts, d, H):
    out, o = {}, 0
    for name, shape in layout(ts, d, H):
        n = int(np.prod(shape))
        out[name] = np.asarray(params[o:o + n], np.float64).reshape(shape)
        o += n
    return out


def forward_backward(params, ts, d, H, X, T):
    """X rows = [u (ts), lam (d)]; loss = 0.5*sum((Y - T)^2).
    Returns (Y, loss, flat gradients)."""
    P = unpack(params, ts, d, H)
    X = np.asarray(X, np.float64)
    T = np.asarray(T, np.float64)
    U, lam = X[:, :ts], X[:, ts:ts + d]
    q = [lam @ P[f"P{l}"] + P[f"p{l}"] for l in (1, 2, 3)]
    g = [gelu(v) for v in q]
    a, h = [], []
    inp = U
    for l in range(3):
        al = inp @ P[f"W{l + 1}"]
        a.append(al)
        h.append(g[l] * al)
        inp = h[-1]
    Y = inp @ P["W4"]
    dY = Y - T
    loss = 0.5 * float(np.sum(dY * dY))
    G = {"W4": h[2].T @ dY}
    dh = dY @ P["W4"].T
    dq = [None] * 3
    for l in (2, 1, 0):
        da = dh * g[l]
        dq[l] = dh * a[l] * dgelu(q[l])
        prev = U if l == 0 else h[l - 1]
        G[f"W{l + 1}"] = prev.T @ da
        dh = da @ P[f"W{l + 1}"].T
    for l in range(3):
        G[f"P{l + 1}"] = lam.T @ dq[l]
        G[f"p{l + 1}"] = dq[l].sum(axis=0)
    flat = np.concatenate([G[name].ravel() for name, _ in layout(ts, d, H)])
    return Y, loss, flat
