"""ORACLE — test infrastructure only.  CPU (numpy, float64) restatement of
the learned quadrature selector's network, its (pair, lag) features and its
convergence labels, the checker for
the device kernels of elastodynamicebem_b200/csrc/selector.cu.  The selector
has no counterpart in the reference.

Parameter layout: W1[64][12], b1[64], W2[64][64], b2[64], W3[4][64], b3[4].
"""
from __future__ import annotations

import numpy as np

F, H, C = 12, 64, 4
SIZES = [("W1", (H, F)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (C, H)), ("b3", (C,))]
NPARAMS = sum(int(np.prod(s)) for _, s in SIZES)


def unpack(params):
    out, k = {}, 0
    p = np.asarray(params, np.float64)
    for name, shape in SIZES:
        n = int(np.prod(shape))
        out[name] = p[k:k + n].reshape(shape)
        k += n
    return out


def loss_and_grad(params, x, y):
    """Mean cross-entropy of softmax(W3 relu(W2 relu(W1 x + b1) + b2) + b3)
    and its gradient (flat, same layout as params)."""
    P = unpack(params)
    x = np.asarray(x, np.float64)
    y = np.asarray(y)
    n = x.shape[0]
    a1 = x @ P["W1"].T + P["b1"]; h1 = np.maximum(a1, 0)
    a2 = h1 @ P["W2"].T + P["b2"]; h2 = np.maximum(a2, 0)
    z = h2 @ P["W3"].T + P["b3"]
    zm = z - z.max(1, keepdims=True)
    pr = np.exp(zm) / np.exp(zm).sum(1, keepdims=True)
    loss = float(np.mean(-np.log(pr[np.arange(n), y])))
    d3 = pr.copy(); d3[np.arange(n), y] -= 1; d3 /= n
    d2 = (d3 @ P["W3"]) * (a2 > 0)
    d1 = (d2 @ P["W2"]) * (a1 > 0)
    g = {"W3": d3.T @ h2, "b3": d3.sum(0), "W2": d2.T @ h1, "b2": d2.sum(0), "W1": d1.T @ x, "b1": d1.sum(0)}
    return loss, np.concatenate([g[name].ravel() for name, _ in SIZES])


def lag_features(mesh, prm, samples):
    """n x 12 features of samples (source, field, lag), as selector.cu
    defines them (lag_features)."""
    samples = np.asarray(samples)
    i, j, l = samples[:, 0], samples[:, 1], samples[:, 2].astype(np.float64)
    c, h, n = mesh.center, mesh.maxL, mesh.normal
    v = c[i] - c[j]
    d = np.maximum(np.linalg.norm(v, axis=1), 0.05 * h[j])
    gap = (d - h[i] - h[j]) / h[j]
    rmin = np.maximum(d - h[i] - h[j], 0.05 * h[j])
    rmax = d + h[i] + h[j]
    tP, tS = prm.velP * l * prm.dt, prm.velS * l * prm.dt
    f = np.zeros((len(samples), F))
    f[:, 0] = np.log(d / h[j]); f[:, 1] = np.log(d / h[i])
    f[:, 2] = np.clip(gap, -2, 20) * 0.1
    f[:, 3] = np.log(h[i] / h[j])
    f[:, 4] = np.abs((n[i] * n[j]).sum(1))
    f[:, 5] = np.abs((n[j] * v).sum(1)) / d
    f[:, 6] = np.abs((n[i] * v).sum(1)) / d
    f[:, 7] = np.minimum(0.1 * tP / rmin, 3.0)
    f[:, 8] = np.minimum(0.1 * tS / rmax, 3.0)
    f[:, 9] = np.clip(0.1 * (tP - d) / h[j], -3.0, 3.0)
    f[:, 10] = np.clip(0.1 * (tS - d) / h[j], -3.0, 3.0)
    f[:, 11] = np.log(prm.velS * prm.dt / h[j])
    return f


def labels(blocks, tol, scale, scales=None):
    """Labels from blocks at the four rules ((4, n, 6)): the smallest rule
    whose block is within tol * scale (times scales[q] when given) of the
    maximal rule's in every entry."""
    blocks = np.asarray(blocks)
    err = np.abs(blocks[:-1] - blocks[-1][None]).max(axis=2)       # (3, n)
    thr = tol * scale * (np.asarray(scales) if scales is not None else 1.0)
    lab = np.full(blocks.shape[1], C - 1)
    for c in range(C - 2, -1, -1):
        lab[err[c] <= thr] = c
    return lab
