"""Test infrastructure: float64 numpy restatement of the learned
preconditioner's network (asgard_b200/csrc/mlp.cu) -- forward pass, MSE loss
and backward pass -- used to check the GPU kernels' gradients.  The network
has no counterpart in the reference; this file is the checker for the
project's own forward/backward kernels, not a product path.

Layout matches asgk_mlp_get_params: per layer W (row-major fan_in x fan_out)
then b, four layers in -> H -> H -> H -> out, GELU (erf form) between.
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


def unpack(params, dims):
    out, o = [], 0
    for l in range(len(dims) - 1):
        nw = dims[l] * dims[l + 1]
        W = params[o:o + nw].reshape(dims[l], dims[l + 1])
        o += nw
        b = params[o:o + dims[l + 1]]
        o += dims[l + 1]
        out.append((W.astype(np.float64), b.astype(np.float64)))
    return out


def forward_backward(params, dims, X, T):
    """loss = 0.5*sum((Y - T)^2); returns (Y, loss, flat gradients)."""
    layers = unpack(np.asarray(params, np.float64), dims)
    X = np.asarray(X, np.float64)
    T = np.asarray(T, np.float64)
    acts, pres = [X], []
    h = X
    for l, (W, b) in enumerate(layers):
        p = h @ W + b
        if l < len(layers) - 1:
            pres.append(p)
            h = gelu(p)
        else:
            h = p
        acts.append(h)
    Y = acts[-1]
    d = Y - T
    loss = 0.5 * float(np.sum(d * d))
    grads = [None] * len(layers)
    dcur = d
    for l in range(len(layers) - 1, -1, -1):
        W, b = layers[l]
        grads[l] = (acts[l].T @ dcur, dcur.sum(axis=0))
        if l == 0:
            break
        dcur = (dcur @ W.T) * dgelu(pres[l - 1])
    flat = np.concatenate([np.concatenate([gW.ravel(), gb]) for gW, gb in grads])
    return Y, loss, flat
