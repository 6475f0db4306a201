"""FP64 restatement of the learned warm start's network, forward and backward (TEST ORACLE ONLY).

Used by tests/ to check the GPU kernels (clothsimulator_b200/csrc/mlp.cu) as the checker, never
by the product.  The network has no counterpart in the reference.  The BF16 rounding points of
the GPU path are reproduced (u1, h1, the aggregated half of u2, h2, the weights, and the BF16
operands dz3, dz2 of the two backward tensor-core products); everything else is FP64, so the
comparison isolates the GPU's FP32 accumulation order.
"""
from __future__ import annotations

import numpy as np

P = 14723
NSTAT = 38
OFF = {"W1": (0, (64, 32)), "b1": (2048, (64,)), "W2": (2112, (64, 128)), "b2": (10304, (64,)),
       "W3": (10368, (64, 64)), "b3": (14464, (64,)), "W4": (14528, (3, 64)), "b4": (14720, (3,))}


def bf16(x):
    """Round to bfloat16 (nearest even) and return as float64."""
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(w):
    w = np.asarray(w, np.float64)
    out = {k: w[o:o + int(np.prod(s))].reshape(s) for k, (o, s) in OFF.items()}
    st = w[P:P + NSTAT]
    out["mu"], out["sigma"], out["mu_y"], out["sigma_y"] = st[:16], st[16:32], st[32:35], st[35:38]
    return out


def neighbours(fx, n):
    """One-ring mesh neighbours (nodes sharing a face), sorted, as the loader builds them."""
    nb = [set() for _ in range(n)]
    for a, b, c in np.asarray(fx):
        nb[a].update((b, c))
        nb[b].update((a, c))
        nb[c].update((a, b))
    return [np.array(sorted(s), np.int64) for s in nb]


def silu(z):
    return z / (1.0 + np.exp(-z))


def silu_grad(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def mean_agg(h, nb):
    return np.stack([h[j].mean(axis=0) if len(j) else np.zeros(h.shape[1]) for j in nb])


def forward(w, feat, nb):
    p = unpack(w)
    W1, W2, W3, W4 = (bf16(p[k]) for k in ("W1", "W2", "W3", "W4"))
    x = (feat - p["mu"]) / p["sigma"]
    u1 = bf16(np.concatenate([x, (mean_agg(feat, nb) - p["mu"]) / p["sigma"]], axis=1))
    z1 = u1 @ W1.T + p["b1"]
    h1 = bf16(silu(z1))
    u2 = np.concatenate([h1, bf16(mean_agg(h1, nb))], axis=1)
    z2 = u2 @ W2.T + p["b2"]
    h2 = bf16(silu(z2))
    z3 = h2 @ W3.T + p["b3"]
    h3 = silu(z3)
    y = h3 @ W4.T + p["b4"]
    return dict(u1=u1, z1=z1, h1=h1, u2=u2, z2=z2, h2=h2, z3=z3, h3=h3, y=y, W2=W2, W3=W3, W4=W4)


def loss_and_grad(w, feat, target, nb):
    """Loss sum_i ||y_i - t_i||^2 / n with t = (target - mu_y) / sigma_y, and its gradient
    with the GPU path's rounding points (straight-through for the roundings)."""
    p = unpack(w)
    f = forward(w, feat, nb)
    n = feat.shape[0]
    t = (target - p["mu_y"]) / p["sigma_y"]
    d = f["y"] - t
    loss = float((d * d).sum() / n)
    return loss, backward(f, 2.0 * d / n, nb), f


def energy_loss_and_grad(w, feat, A, b, dv_star, node_ranges, nb):
    """Energy-norm loss of the prediction p = previous dv + sigma_y y + mu_y (the previous dv is
    features 12-14): the mean over sheets of sin^2 of the angle between p and dv* in the A inner
    product, 1 - u^2 / (w c) with u = p^T b, w = p^T A p, c = dv*^T b (A dv* = b), and its
    gradient through dL/dp = (2 u / (w c S)) (u / w A p - b).  A: the batch's 3N x 3N matrix
    (SciPy), b and dv* 3N vectors, node_ranges the sheets' (first node, end) pairs."""
    p = unpack(w)
    f = forward(w, feat, nb)
    pred = feat[:, 12:15] + p["sigma_y"] * f["y"] + p["mu_y"]
    pv = pred.reshape(-1)
    Ap = A @ pv
    S = len(node_ranges)
    dp = np.zeros_like(pv)
    loss = 0.0
    for n0, n1 in node_ranges:
        sl = slice(3 * n0, 3 * n1)
        c = float(dv_star[sl] @ b[sl])
        u = float(pv[sl] @ b[sl])
        ww = float(pv[sl] @ Ap[sl])
        loss += (1.0 - u * u / (ww * c)) / S
        dp[sl] = 2.0 * u / (ww * c * S) * (u / ww * Ap[sl] - b[sl])
    dy = dp.reshape(-1, 3) * p["sigma_y"]
    return loss, backward(f, dy, nb), pred


def backward(f, dy, nb):
    """Gradient of the weights (flat, P floats) from dL/dy, with the GPU path's rounding points."""
    g = {}
    g["W4"] = dy.T @ f["h3"]
    g["b4"] = dy.sum(0)
    dz3 = (dy @ f["W4"]) * silu_grad(f["z3"])
    g["W3"] = dz3.T @ f["h2"]
    g["b3"] = dz3.sum(0)
    dh2 = bf16(dz3) @ f["W3"]
    dz2 = dh2 * silu_grad(f["z2"])
    g["W2"] = dz2.T @ f["u2"]
    g["b2"] = dz2.sum(0)
    du2 = bf16(dz2) @ f["W2"]
    dh1 = du2[:, :64].copy()
    deg = np.array([len(j) for j in nb], np.float64)
    for i, js in enumerate(nb):
        for j in js:
            dh1[i] += du2[j, 64:] / deg[j]
    dz1 = dh1 * silu_grad(f["z1"])
    g["W1"] = dz1.T @ f["u1"]
    g["b1"] = dz1.sum(0)
    flat = np.zeros(P)
    for k, (o, s) in OFF.items():
        flat[o:o + int(np.prod(s))] = g[k].reshape(-1)
    return flat


def predict(w, feat, nb):
    p = unpack(w)
    f = forward(w, feat, nb)
    return feat[:, 12:15] + p["sigma_y"] * f["y"] + p["mu_y"]
