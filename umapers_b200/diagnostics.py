"""Quality metrics used to assess embeddings.

``trustworthiness_report`` mirrors umap_rs/python/umapers/diagnostics.py:1-53
(sklearn's trustworthiness).  ``knn_preservation`` is the kNN-recall measure of
benchmarks/compare_real_impls_fair.py:455-530: the mean fraction of each
row's k nearest neighbours in the input that are also among its k nearest
neighbours in the embedding.
"""
from __future__ import annotations

from typing import Any

import numpy as np


def _as_2d_f32(x: Any, name: str) -> np.ndarray:
    arr = np.asarray(x, dtype=np.float32)
    if arr.ndim != 2:
        raise ValueError(f"{name} must be a 2D array, got ndim={arr.ndim}")
    return arr


def trustworthiness_report(data: Any, model_or_embedding: Any, *, n_neighbors: int = 15) -> dict:
    """Return a compact nearest-neighbor preservation report."""
    if n_neighbors < 1:
        raise ValueError("n_neighbors must be >= 1")
    from sklearn.manifold import trustworthiness

    x = _as_2d_f32(data, "data")
    emb = _as_2d_f32(getattr(model_or_embedding, "embedding_", model_or_embedding), "embedding")
    if x.shape[0] != emb.shape[0]:
        raise ValueError("data and embedding row counts must match")
    score = float(trustworthiness(x, emb, n_neighbors=n_neighbors))
    return {
        "trustworthiness": score,
        "n_samples": int(x.shape[0]),
        "n_features": int(x.shape[1]),
        "n_components": int(emb.shape[1]),
        "n_neighbors": int(n_neighbors),
    }


def _knn_sets(x: np.ndarray, k: int) -> np.ndarray:
    from sklearn.neighbors import NearestNeighbors

    nn = NearestNeighbors(n_neighbors=k + 1, algorithm="brute").fit(x)
    idx = nn.kneighbors(x, return_distance=False)
    return idx[:, 1:]


def knn_preservation(data: Any, embedding: Any, *, n_neighbors: int = 15) -> float:
    """Mean overlap of input-space and embedding-space k-NN sets."""
    x = _as_2d_f32(data, "data").astype(np.float64)
    e = _as_2d_f32(embedding, "embedding").astype(np.float64)
    a = _knn_sets(x, n_neighbors)
    b = _knn_sets(e, n_neighbors)
    hits = [len(set(a[i]).intersection(b[i])) for i in range(a.shape[0])]
    return float(np.mean(hits) / n_neighbors)


def quality(data: Any, embedding: Any, *, n_neighbors: int = 15, sample: int | None = 10_000,
            seed: int = 0) -> dict[str, float]:
    """trustworthiness@k and k-NN preservation on a fixed random subset with
    neighbours recomputed on that subset."""
    x = _as_2d_f32(data, "data")
    e = _as_2d_f32(embedding, "embedding")
    n = x.shape[0]
    if sample is not None and n > sample:
        rows = np.sort(np.random.default_rng(seed).choice(n, size=sample, replace=False))
        x, e = x[rows], e[rows]
    from sklearn.manifold import trustworthiness

    return {
        "trustworthiness": float(trustworthiness(x, e, n_neighbors=n_neighbors)),
        "knn_preservation": knn_preservation(x, e, n_neighbors=n_neighbors),
    }
