"""CPU checks of the surrogate's FP64 oracle (oracle/mlp.py) and host-side
surface: the oracle's analytic gradients against finite differences, its
bfloat16 rounding against torch's, and the Python options plumbing."""
import numpy as np
import pytest
import torch

from oracle import mlp


def _problem(rng, B=6, din=5, hidden=8, n_out=2, n_teacher=20, n_neg=0, scale=0.3):
    x = rng.normal(size=(B, din))
    params = mlp.glorot(rng, din, hidden, n_out)
    targets = rng.normal(scale=scale, size=(B, n_out))
    teacher = rng.normal(scale=scale, size=(n_teacher, n_out))
    counts = rng.integers(0, 4, size=B)
    edge_ptr = np.concatenate([[0], np.cumsum(counts)])
    edge_tail = rng.integers(0, n_teacher, size=edge_ptr[-1])
    edge_weight = rng.uniform(0.1, 1.0, size=edge_ptr[-1])
    neg_tail = rng.integers(0, n_teacher, size=(B, n_neg))
    return x, params, targets, teacher, edge_ptr, edge_tail, edge_weight, neg_tail


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    x, params, targets, teacher, ep, et, ew, nt = _problem(rng)
    kw = dict(a=1.577, b=0.895, mse_w=1.0, edge_w=0.5, neg_scale=5.0, hidden=8, n_out=2,
              rounding=False)

    def loss_of(p):
        return mlp.forward_backward(x, targets, p, teacher, ep, et, ew, nt, **kw)[1]

    g, _, y = mlp.forward_backward(x, targets, params, teacher, ep, et, ew, nt, **kw)
    # the clip of the attractive pair term stays inactive at these scales
    h = 1e-6
    fd = np.empty_like(params)
    for i in range(params.size):
        e = np.zeros_like(params)
        e[i] = h
        fd[i] = (loss_of(params + e) - loss_of(params - e)) / (2 * h)
    err = np.abs(fd - g).max() / np.abs(g).max()
    assert err < 1e-6, err


def test_repulsive_gradient_is_the_reference_sgd_form():
    # one row, one negative, no edges: g = edge_w / B * rep_w * clip(c * diff)
    y = np.array([[0.3, -0.2]])
    teacher = np.array([[0.0, 0.0]])
    a, b = 1.577, 0.895
    g, _ = mlp.loss_grad(y, y, teacher, [0, 1], [0], [2.0], [[0]], a, b, 0.0, 1.0, 5.0)
    d2 = 0.13
    c = -2 * b / ((0.001 + d2) * (1 + a * d2 ** b))
    expected = 5.0 * 2.0 / 1 * np.clip(c * y[0], -4, 4)
    # the attractive edge to the same point also contributes
    ca = 2 * a * b * d2 ** b / (d2 * (1 + a * d2 ** b))
    expected = expected + 2.0 * np.clip(ca * y[0], -4, 4)
    assert np.allclose(g[0], expected, rtol=1e-12)


def test_bf16_rounding_matches_torch():
    rng = np.random.default_rng(1)
    v = np.concatenate([rng.normal(scale=s, size=2000) for s in (1e-3, 1.0, 1e3)])
    v = np.concatenate([v, [1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -0.0, 65504.0, 1e-30]])
    ours = mlp.bf16(v)
    theirs = torch.tensor(v.astype(np.float32)).to(torch.bfloat16).to(torch.float64).numpy()
    assert np.array_equal(ours, theirs)


def test_standardize_follows_the_parametric_rule():
    x = np.array([[1.0, 5.0], [3.0, 5.0], [5.0, 5.0]], np.float32)
    mean, scale, xs = mlp.standardize(x)
    assert np.allclose(mean, [3.0, 5.0])
    assert np.allclose(scale, [np.sqrt(8.0 / 3.0), 1.0])  # constant column keeps scale 1
    assert np.allclose(xs[:, 1], 0.0)


def test_umap_surrogate_options_are_validated():
    from umapers import Umap

    with pytest.raises(ValueError, match="transform_mode"):
        Umap(transform_mode="learned")
    m = Umap(transform_mode="surrogate", surrogate_kwds={"epochs": 2})
    assert m.get_params()["transform_mode"] == "surrogate"
    assert m.get_params()["surrogate_kwds"] == {"epochs": 2}
    with pytest.raises(ValueError, match="method must be one of"):
        m.transform(np.zeros((2, 3), np.float32), method="learned")


def test_surrogate_before_fit_raises():
    from umapers import Umap

    m = Umap()
    with pytest.raises(RuntimeError, match="not fitted"):
        m.fit_surrogate()
    with pytest.raises(ValueError, match="unknown surrogate option"):
        m._core.fit_surrogate(hiddne=3)
