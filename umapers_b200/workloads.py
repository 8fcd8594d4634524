"""Seeded synthetic inputs with the shapes and distributions of the
benchmark configurations, and the deterministic generators of the reference's
unit tests.  No public dataset is involved; every generator uses
``numpy.random.default_rng(seed)`` and returns C-contiguous float32.
"""
from __future__ import annotations

import numpy as np


def gaussian(n: int = 1000, d: int = 32, seed: int = 42) -> np.ndarray:
    """i.i.d. N(0, 1) rows (the 1000 x 32 quick-start configuration)."""
    return np.random.default_rng(seed).normal(size=(n, d)).astype(np.float32)


def isotropic_mixture(n: int, d: int, n_comp: int, mean_std: float, seed: int,
                      return_labels: bool = False):
    """Equal-weight mixture of unit-variance Gaussians with means ~ N(0, mean_std^2)
    (the 20 000 x 192, 10-component configuration uses mean_std=4, seed 7)."""
    rng = np.random.default_rng(seed)
    means = rng.normal(0.0, mean_std, size=(n_comp, d))
    labels = rng.integers(0, n_comp, size=n)
    x = (means[labels] + rng.normal(size=(n, d))).astype(np.float32)
    return (x, labels) if return_labels else x


def anisotropic_mixture(n: int = 1_000_000, d: int = 64, n_comp: int = 50, seed: int = 11,
                        return_labels: bool = False):
    """Equal-weight mixture of axis-aligned Gaussians: means ~ N(0, 5^2),
    per-component per-dim std ~ U(0.5, 2) (the 1M x 64 configuration)."""
    rng = np.random.default_rng(seed)
    means = rng.normal(0.0, 5.0, size=(n_comp, d))
    stds = rng.uniform(0.5, 2.0, size=(n_comp, d))
    labels = rng.integers(0, n_comp, size=n)
    x = np.empty((n, d), dtype=np.float32)
    chunk = 1 << 18
    for s in range(0, n, chunk):
        lab = labels[s:s + chunk]
        x[s:s + chunk] = means[lab] + stds[lab] * rng.normal(size=(lab.shape[0], d))
    return (x, labels) if return_labels else x


def transform_mixture(n_fit: int = 200_000, n_query: int = 1_000_000, d: int = 128,
                      n_comp: int = 20, seed: int = 5, query_seed: int = 6):
    """Fit rows and query rows from the same 20-component mixture (means
    ~ N(0, 4^2), unit variance); queries are drawn with their own seed."""
    rng = np.random.default_rng(seed)
    means = rng.normal(0.0, 4.0, size=(n_comp, d))
    lab = rng.integers(0, n_comp, size=n_fit)
    fit = (means[lab] + rng.normal(size=(n_fit, d))).astype(np.float32)
    qrng = np.random.default_rng(query_seed)
    qlab = qrng.integers(0, n_comp, size=n_query)
    query = (means[qlab] + qrng.normal(size=(n_query, d))).astype(np.float32)
    return fit, query


def reference_synthetic(n: int, dim: int) -> np.ndarray:
    """The two-cluster sin/cos generator of the reference tests
    (rust_umap/src/lib.rs:5752-5765), evaluated in float32."""
    i = np.arange(n, dtype=np.float32)[:, None]
    dd = np.arange(dim, dtype=np.float32)[None, :]
    t = (i + np.float32(1.3) * dd) / np.float32(n)
    shift = np.where(np.arange(n) < n // 2, 0.0, 5.0).astype(np.float32)[:, None]
    x = shift + np.sin(np.float32(10.0) * t) * np.float32(0.2) + np.cos(np.float32(7.0) * t) * np.float32(0.1)
    return x.astype(np.float32)


def disconnected_components(n_components: int, points_per_component: int):
    """Rings far apart in the first coordinate (rust_umap/src/lib.rs:5862-5888)."""
    rows, labels = [], []
    for c in range(n_components):
        shift = c * 50.0
        for p in range(points_per_component):
            t = 2.0 * np.pi * p / points_per_component
            rows.append([shift + np.cos(t), np.sin(t), np.cos(2 * t), np.sin(2 * t),
                         -1.0 + 2.0 * p / points_per_component, c * 0.1, 0.0, 0.0])
            labels.append(c)
    return np.asarray(rows, dtype=np.float32), np.asarray(labels)


def three_centres(n_samples: int = 180, n_features: int = 12, seed: int = 42) -> np.ndarray:
    """Three-centre standardised dataset of the reference binding tests
    (umap_rs/tests/test_binding.py:27-41)."""
    rng = np.random.default_rng(seed)
    centers = np.stack([
        np.linspace(-2.0, 2.0, n_features, dtype=np.float32),
        np.linspace(1.5, -1.5, n_features, dtype=np.float32),
        np.zeros(n_features, dtype=np.float32),
    ])
    labels = rng.integers(0, len(centers), size=n_samples)
    noise = rng.normal(0.0, 0.35, size=(n_samples, n_features)).astype(np.float32)
    x = centers[labels] + noise
    x -= x.mean(axis=0, keepdims=True)
    x /= x.std(axis=0, keepdims=True) + 1e-6
    return x.astype(np.float32)


def sparse_lognormal_csr(n: int = 200_000, d: int = 2000, nnz_row: int = 20, seed: int = 3):
    """CSR rows with about `nnz_row` stored values each: column positions
    drawn uniformly per row (repeats merged, so a row holds at most
    `nnz_row`), sorted, values LogNormal(0, 1) (the sparse text-like
    configuration, 200,000 x 2,000 at 1%)."""
    import scipy.sparse as sp

    rng = np.random.default_rng(seed)
    cols = np.sort(rng.integers(0, d, size=(n, nnz_row)), axis=1)
    keep = np.ones_like(cols, dtype=bool)
    keep[:, 1:] = cols[:, 1:] != cols[:, :-1]
    counts = keep.sum(axis=1)
    indptr = np.zeros(n + 1, np.int64)
    np.cumsum(counts, out=indptr[1:])
    indices = cols[keep].astype(np.int64)
    data = rng.lognormal(0.0, 1.0, size=indices.shape[0]).astype(np.float32)
    return sp.csr_matrix((data, indices, indptr), shape=(n, d))
