"""CPU FP64 oracle of the transform surrogate's network and loss.

Test infrastructure only: the tests and smoke() use it as the checker of
umapb_mlp_grad (umapers_b200/csrc/surrogate.cu); nothing in the product path
imports it.

The surrogate has no reference function.  Its precedent is the reference's
ParametricUmapModel (rust_umap/src/parametric.rs:89-534), whose input
standardisation rule (parametric.rs:652-675: scale = std when std > 1e-6,
else 1) is restated by `standardize`.  The loss's pair terms follow the
reference's SGD: the attractive coefficient 2ab d^(2b-2) / (1 + a d^(2b))
(rust_umap/src/lib.rs:5170, 5193-5194), the repulsive one
-2b / ((0.001 + d^2)(1 + a d^(2b))) (lib.rs:5225-5229), each coordinate
clipped to [-4, 4] (clip, lib.rs:4962-4964).

`rounding=True` rounds to bfloat16 at the points where the GPU stores bf16
(the standardised input, W1, W2, both hidden activations and both hidden
gradients) and computes everything else in FP64, so the GPU's gradients
differ from it only by FP32 accumulation.  `rounding=False` is the exact
network, whose gradients tests check against finite differences.
"""
from __future__ import annotations

import numpy as np
from scipy.special import erf

SCALE_EPS = 1e-6


def bf16(x) -> np.ndarray:
    """Round to bfloat16 (round to nearest even on the FP32 value)."""
    f = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_grad(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def standardize(x: np.ndarray):
    """Per-feature mean and scale (parametric.rs:652-675) and the scaled rows."""
    x64 = np.asarray(x, np.float64)
    mean = x64.mean(axis=0)
    std = np.sqrt(np.maximum((x64 * x64).mean(axis=0) - mean * mean, 0.0))
    scale = np.where(std > SCALE_EPS, std, 1.0)
    return mean, scale, (x64 - mean) / scale


def layout(n_features: int, hidden: int, n_out: int) -> dict:
    """Offsets of W1, b1, W2, b2, W3, b3 in the flat parameter vector."""
    sizes = [("W1", hidden * n_features), ("b1", hidden), ("W2", hidden * hidden),
             ("b2", hidden), ("W3", n_out * hidden), ("b3", n_out)]
    out, off = {}, 0
    for name, size in sizes:
        out[name] = (off, size)
        off += size
    out["total"] = off
    return out


def unpack(params: np.ndarray, n_features: int, hidden: int, n_out: int) -> dict:
    lay = layout(n_features, hidden, n_out)
    p = np.asarray(params, np.float64)
    shapes = {"W1": (hidden, n_features), "b1": (hidden,), "W2": (hidden, hidden),
              "b2": (hidden,), "W3": (n_out, hidden), "b3": (n_out,)}
    return {k: p[lay[k][0]:lay[k][0] + lay[k][1]].reshape(shapes[k]) for k in shapes}


def pack(parts: dict, n_features: int, hidden: int, n_out: int) -> np.ndarray:
    lay = layout(n_features, hidden, n_out)
    out = np.zeros(lay["total"], np.float64)
    for k in ("W1", "b1", "W2", "b2", "W3", "b3"):
        off, size = lay[k]
        out[off:off + size] = np.asarray(parts[k], np.float64).reshape(-1)
    return out


def loss_grad(y, targets, teacher, edge_ptr, edge_tail, edge_weight, neg_tail, a, b, mse_w,
              edge_w, neg_scale):
    """Batch-mean loss and its gradient with respect to the outputs y (B x n_out)."""
    y = np.asarray(y, np.float64)
    B = y.shape[0]
    teacher = np.asarray(teacher, np.float64)
    r = y - np.asarray(targets, np.float64)
    g = 2.0 * mse_w / B * r
    loss = mse_w * float((r * r).sum())
    counts = np.diff(np.asarray(edge_ptr, np.int64))
    rows = np.repeat(np.arange(B), counts)
    w = np.asarray(edge_weight, np.float64)
    if rows.size:
        diff = y[rows] - teacher[np.asarray(edge_tail, np.int64)]
        d2 = (diff * diff).sum(axis=1)
        pos = d2 > 0.0
        db = np.where(pos, np.power(np.where(pos, d2, 1.0), b), 0.0)
        c = np.where(pos, 2.0 * a * b * db / (np.where(pos, d2, 1.0) * (1.0 + a * db)), 0.0)
        np.add.at(g, rows, (edge_w / B) * w[:, None] * np.clip(c[:, None] * diff, -4.0, 4.0))
        loss += edge_w * float((w * np.log1p(a * db) * pos).sum())
    wsum = np.bincount(rows, weights=w, minlength=B) if rows.size else np.zeros(B)
    neg_tail = np.asarray(neg_tail, np.int64).reshape(B, -1)
    n_neg = neg_tail.shape[1]
    if n_neg > 0:
        rep_w = neg_scale * wsum / n_neg
        diff = y[:, None, :] - teacher[neg_tail]
        d2 = (diff * diff).sum(axis=2)
        db = np.where(d2 > 0.0, np.power(np.maximum(d2, 0.0), b), 0.0)
        c = -2.0 * b / ((0.001 + d2) * (1.0 + a * db))
        g += (edge_w / B) * rep_w[:, None] * np.clip(c[..., None] * diff, -4.0, 4.0).sum(axis=1)
        loss += edge_w * float((rep_w[:, None] * np.log1p(1.0 / (a * db + 1e-6))).sum())
    return g, loss / B


def forward_backward(x, targets, params, teacher, edge_ptr, edge_tail, edge_weight, neg_tail,
                     a, b, mse_w, edge_w, neg_scale, hidden, n_out, rounding=True,
                     out_shift=None, out_scale=None):
    """Flat gradient (same layout as params), batch-mean loss and outputs
    y = out_shift + out_scale * (a2 W3^T + b3)."""
    rnd = bf16 if rounding else (lambda v: np.asarray(v, np.float64))
    x = np.asarray(x, np.float64)
    n_features = x.shape[1]
    p = unpack(params, n_features, hidden, n_out)
    xb = rnd(x)
    w1, w2, w3 = rnd(p["W1"]), rnd(p["W2"]), p["W3"]
    z1 = xb @ w1.T + p["b1"]
    a1 = rnd(gelu(z1))
    z2 = a1 @ w2.T + p["b2"]
    a2 = rnd(gelu(z2))
    shift = np.zeros(n_out) if out_shift is None else np.asarray(out_shift, np.float64)
    scale = np.ones(n_out) if out_scale is None else np.asarray(out_scale, np.float64)
    y = shift + scale * (a2 @ w3.T + p["b3"])
    dy, loss = loss_grad(y, targets, teacher, edge_ptr, edge_tail, edge_weight, neg_tail, a, b,
                         mse_w, edge_w, neg_scale)
    dy = dy * scale
    dz2 = rnd((dy @ w3) * gelu_grad(z2))
    dz1 = rnd((dz2 @ w2) * gelu_grad(z1))
    grads = {
        "W3": dy.T @ a2, "b3": dy.sum(axis=0),
        "W2": dz2.T @ a1, "b2": dz2.sum(axis=0),
        "W1": dz1.T @ xb, "b1": dz1.sum(axis=0),
    }
    return pack(grads, n_features, hidden, n_out), loss, y


def glorot(rng: np.random.Generator, n_features: int, hidden: int, n_out: int) -> np.ndarray:
    """Glorot-uniform weights and zero biases (the limit of parametric.rs:190-208)."""
    def u(rows, cols):
        lim = np.sqrt(6.0 / (rows + cols))
        return rng.uniform(-lim, lim, size=(rows, cols))
    parts = {"W1": u(hidden, n_features), "b1": np.zeros(hidden),
             "W2": u(hidden, hidden), "b2": np.zeros(hidden),
             "W3": u(n_out, hidden), "b3": np.zeros(n_out)}
    return pack(parts, n_features, hidden, n_out)
