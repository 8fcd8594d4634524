"""The ``Umap`` estimator and module-level ``fit_transform``.

Same public surface as the reference's Python facade (umap_rs/python/umapers/
_api.py:324-873, 1054-1094): keyword arguments and defaults, sklearn-style
``get_params``/``set_params``, array normalisation (C-contiguous float32,
int64 kNN indices), ``out=`` buffers, the ``ann_mode`` shortcut, and the
fitted attributes ``embedding_``, ``n_features_in_``, ``n_samples_fit_``.
Compute runs on one B200 through ``UmapCore`` (libumapb200.so), densMAP and
``output_dens`` (dense input), categorical supervision (``target_metric=
"categorical"`` with ``y``, dense input) and CSR sparse input (scipy
csr/csc/coo) included, and ``inverse_transform`` of dense-fitted models.
Inputs the engine does not cover (metrics other than euclidean/cosine, sparse
input with n_neighbors above 32) raise ValueError.
"""
from __future__ import annotations

from typing import Any, TypedDict

import numpy as np

from ._umapers import AlignedUmapCore, ParametricUmapCore, UmapCore

_PARAM_NAMES = (
    "n_neighbors",
    "n_components",
    "n_epochs",
    "metric",
    "metric_kwds",
    "learning_rate",
    "min_dist",
    "spread",
    "local_connectivity",
    "set_op_mix_ratio",
    "repulsion_strength",
    "negative_sample_rate",
    "random_seed",
    "init",
    "ann_mode",
    "use_approximate_knn",
    "approx_knn_candidates",
    "approx_knn_iters",
    "approx_knn_threshold",
    "densmap",
    "dens_lambda",
    "dens_frac",
    "dens_var_shift",
    "output_dens",
    "target_metric",
    "target_weight",
    "target_n_neighbors",
    "knn_backend",
    "transform_mode",
    "surrogate_kwds",
)

_TRANSFORM_MODES = ("plain", "surrogate")

_FITTED_ATTRS = (
    "embedding_",
    "n_features_in_",
    "n_samples_fit_",
    "radii_original_",
    "radii_embedding_",
    "rad_orig_",
    "rad_emb_",
    "knn_diagnostics_",
    "surrogate_info_",
    "transform_fallback_",
)

_METRIC_ALIASES = {
    "euclidean": "euclidean",
    "l2": "euclidean",
    "manhattan": "manhattan",
    "l1": "manhattan",
    "cosine": "cosine",
    "chebyshev": "chebyshev",
    "linfinity": "chebyshev",
    "linf": "chebyshev",
    "minkowski": "minkowski",
    "correlation": "correlation",
    "canberra": "canberra",
    "braycurtis": "braycurtis",
    "bray_curtis": "braycurtis",
}


class UmapKwargs(TypedDict, total=False):
    """Keyword arguments accepted by ``Umap(...)`` and ``fit_transform(..., **kwargs)``."""

    n_neighbors: int
    n_components: int
    n_epochs: int | None
    metric: str
    metric_kwds: dict[str, Any] | None
    learning_rate: float
    min_dist: float
    spread: float
    local_connectivity: float
    set_op_mix_ratio: float
    repulsion_strength: float
    negative_sample_rate: int
    random_seed: int
    init: str
    ann_mode: str
    use_approximate_knn: bool
    approx_knn_candidates: int
    approx_knn_iters: int
    approx_knn_threshold: int
    densmap: bool
    dens_lambda: float
    dens_frac: float
    dens_var_shift: float
    output_dens: bool
    target_metric: str | None
    target_weight: float
    target_n_neighbors: int | None
    knn_backend: str


def _f32_matrix(x: Any, name: str) -> np.ndarray:
    arr = np.asarray(x, dtype=np.float32, order="C")
    if arr.ndim != 2:
        raise ValueError(f"{name} must be a 2D array, got ndim={arr.ndim}")
    return arr


def _i64_matrix(x: Any, name: str) -> np.ndarray:
    arr = np.asarray(x, dtype=np.int64, order="C")
    if arr.ndim != 2:
        raise ValueError(f"{name} must be a 2D array, got ndim={arr.ndim}")
    return arr


def _is_sparse(x: Any) -> bool:
    return getattr(x, "format", None) in {"csr", "csc", "coo"}


def _maybe_as_csr_parts(x: Any, name: str):
    """(indptr, indices, data, n_rows, n_cols) of a scipy-style sparse matrix
    in canonical CSR form, or None for dense input (the reference facade's
    _maybe_as_csr_parts, umapers/_api.py:143-190)."""
    fmt = getattr(x, "format", None)
    if fmt == "csr":
        matrix = x
    elif fmt in {"csc", "coo"}:
        tocsr = getattr(x, "tocsr", None)
        if not callable(tocsr):
            raise ValueError(f"{name} sparse input with format={fmt!r} cannot be converted to CSR")
        matrix = tocsr()
        if getattr(matrix, "format", None) != "csr":
            raise ValueError(f"{name}.tocsr() must return a CSR matrix")
    else:
        return None
    if getattr(matrix, "has_canonical_format", True) is False:
        matrix = matrix.copy()
        matrix.sum_duplicates()
        matrix.sort_indices()
    elif getattr(matrix, "has_sorted_indices", True) is False:
        matrix = matrix.copy()
        matrix.sort_indices()
    shape = getattr(matrix, "shape", None)
    if shape is None or len(shape) != 2:
        raise ValueError(f"{name} must be a 2D CSR matrix")
    n_rows, n_cols = int(shape[0]), int(shape[1])
    if n_cols <= 0:
        raise ValueError(f"{name} must have at least one column")
    indptr = np.asarray(matrix.indptr, dtype=np.int64, order="C")
    indices = np.asarray(matrix.indices, dtype=np.int64, order="C")
    data = np.asarray(matrix.data, dtype=np.float32, order="C")
    if indptr.ndim != 1 or indices.ndim != 1 or data.ndim != 1:
        raise ValueError(f"{name} CSR arrays must be 1D")
    if indices.shape[0] != data.shape[0]:
        raise ValueError(f"{name} CSR indices/data length mismatch")
    return indptr, indices, data, n_rows, n_cols


def _out_buffer(out: Any, shape: tuple[int, int]) -> np.ndarray:
    """Output-buffer contract of the reference (_api.py:193-206)."""
    if not isinstance(out, np.ndarray):
        raise TypeError("out must be a NumPy ndarray")
    if out.dtype != np.float32:
        raise TypeError(f"out dtype must be float32, got {out.dtype}")
    if out.ndim != 2:
        raise ValueError(f"out must be 2D, got ndim={out.ndim}")
    if not out.flags.c_contiguous:
        raise ValueError("out must be C-contiguous")
    if not out.flags.writeable:
        raise ValueError("out must be writeable")
    if tuple(out.shape) != tuple(shape):
        raise ValueError(f"output buffer shape mismatch: expected {shape}, got {tuple(out.shape)}")
    return out


def _ann_mode(ann_mode: Any, use_approx: bool, threshold: int) -> tuple[str, bool, int]:
    """ann_mode shortcut (_api.py:209-224): exact forces the exact kNN,
    approximate forces NN-descent for every input size.  A canonical value is
    kept as the same object, so sklearn's clone sees the parameter unchanged."""
    if isinstance(ann_mode, str) and ann_mode in ("auto", "exact", "approximate"):
        mode = ann_mode
    else:
        mode = str(ann_mode).lower()
    if mode == "auto":
        return mode, use_approx, threshold
    if mode == "exact":
        return mode, False, threshold
    if mode == "approximate":
        return mode, True, 0
    raise ValueError(f"unsupported ann_mode '{ann_mode}', expected auto|exact|approximate")


def _as_labels(x: Any, name: str) -> np.ndarray:
    """Class labels as a C-contiguous int64 vector (_api.py:127-131)."""
    arr = np.asarray(x, dtype=np.int64, order="C")
    if arr.ndim != 1:
        raise ValueError(f"{name} must be a 1D label array, got ndim={arr.ndim}")
    return arr


def _target_metric(target_metric: Any) -> str | None:
    if target_metric is None:
        return None
    metric = str(target_metric).lower()
    if metric in {"none", ""}:
        return None
    if metric == "categorical":
        return target_metric if target_metric == metric else metric
    raise ValueError(f"unsupported target_metric '{target_metric}', expected None|categorical")


def _metric_config(metric: Any, metric_kwds: Any) -> tuple[str, Any, float | None]:
    name = str(metric).lower()
    if name not in _METRIC_ALIASES:
        expected = "|".join(sorted(set(_METRIC_ALIASES.values())))
        raise ValueError(f"unsupported metric '{metric}', expected {expected}")
    name = _METRIC_ALIASES[name]
    if isinstance(metric, str) and metric == name:
        name = metric  # keep the caller's object (sklearn's clone compares identity)
    kwds = {} if metric_kwds is None else metric_kwds
    if not hasattr(kwds, "keys"):
        raise TypeError("metric_kwds must be a mapping or None")
    keys = set(kwds.keys())
    if name == "minkowski":
        if "p" not in keys:
            raise ValueError("metric='minkowski' requires metric_kwds={'p': ...}")
        extra = keys - {"p"}
        if extra:
            raise ValueError(
                f"unsupported metric_kwds for minkowski: {', '.join(sorted(map(str, extra)))}"
            )
        p = float(kwds["p"])
        if not np.isfinite(p) or p <= 0.0:
            raise ValueError("metric_kwds['p'] must be finite and > 0 for minkowski")
        return name, metric_kwds, p
    if keys:
        raise ValueError(f"unsupported metric_kwds for {name}: {', '.join(sorted(map(str, keys)))}")
    return name, metric_kwds, None


def _dens_params(lam: float, frac: float, shift: float) -> tuple[float, float, float]:
    lam, frac, shift = float(lam), float(frac), float(shift)
    if not np.isfinite(lam) or lam < 0.0:
        raise ValueError("dens_lambda must be finite and >= 0")
    if not np.isfinite(frac) or frac < 0.0 or frac > 1.0:
        raise ValueError("dens_frac must be finite and in [0, 1]")
    if not np.isfinite(shift) or shift <= 0.0:
        raise ValueError("dens_var_shift must be finite and > 0")
    return lam, frac, shift


class Umap:
    """UMAP estimator running on one NVIDIA B200.

    The estimator keeps the reference package's surface: array-like input is
    normalised to a C-contiguous ``float32`` matrix and forwarded to the CUDA
    engine; ``fit`` stores the training matrix and embedding on the device
    so ``transform`` can place new rows.

    Example
    -------
    >>> import numpy as np
    >>> from umapers import Umap
    >>> x = np.random.default_rng(42).normal(size=(100, 8)).astype(np.float32)
    >>> emb = Umap(n_neighbors=15, n_components=2).fit_transform(x)
    """

    def __init__(
        self,
        *,
        n_neighbors: int = 15,
        n_components: int = 2,
        n_epochs: int | None = None,
        metric: str = "euclidean",
        metric_kwds: dict[str, Any] | None = None,
        learning_rate: float = 1.0,
        min_dist: float = 0.1,
        spread: float = 1.0,
        local_connectivity: float = 1.0,
        set_op_mix_ratio: float = 1.0,
        repulsion_strength: float = 1.0,
        negative_sample_rate: int = 5,
        random_seed: int = 42,
        init: str = "spectral",
        ann_mode: str = "auto",
        use_approximate_knn: bool = True,
        approx_knn_candidates: int = 50,
        approx_knn_iters: int = 14,
        approx_knn_threshold: int = 4096,
        densmap: bool = False,
        dens_lambda: float = 2.0,
        dens_frac: float = 0.3,
        dens_var_shift: float = 0.1,
        output_dens: bool = False,
        target_metric: str | None = None,
        target_weight: float = 0.5,
        target_n_neighbors: int | None = None,
        knn_backend: str = "auto",
        transform_mode: str = "plain",
        surrogate_kwds: dict[str, Any] | None = None,
    ) -> None:
        """Create a UMAP model.

        Parameters
        ----------
        n_neighbors:
            Number of neighbors used to build the neighborhood graph.
        n_components:
            Output embedding dimension.
        n_epochs:
            Number of optimization epochs; ``None`` uses 500 for up to 10 000
            samples and 200 above (transform: 100 / 30).
        metric, metric_kwds:
            Distance metric.  The GPU engine computes euclidean and cosine.
        learning_rate, min_dist, spread, local_connectivity, set_op_mix_ratio,
        repulsion_strength, negative_sample_rate, random_seed, init:
            Standard UMAP hyperparameters.
        ann_mode:
            ``auto`` | ``exact`` | ``approximate`` shortcut over the two
            flags below.
        use_approximate_knn, approx_knn_candidates, approx_knn_iters,
        approx_knn_threshold:
            NN-descent switch and tuning.
        densmap, dens_lambda, dens_frac, dens_var_shift, output_dens:
            densMAP controls.  With ``output_dens``, ``fit_transform`` returns
            ``(embedding, radii_original, radii_embedding)``.
        target_metric, target_weight, target_n_neighbors:
            Supervised-target controls (validated; the GPU engine fits
            unsupervised).
        knn_backend:
            ``auto`` | ``tensor`` | ``plain``: how exact-kNN tiles are
            computed; every backend returns the same neighbours.
        transform_mode:
            ``plain`` (the reference's kNN + SGD transform) or ``surrogate``:
            every fit also trains a BF16 MLP that maps rows straight to the
            embedding, and ``transform`` uses it, sending the rows its gate
            rejects to the plain transform.
        surrogate_kwds:
            Options of the surrogate (see ``UmapCore.fit_surrogate``).
        """
        for attr in _FITTED_ATTRS:
            if hasattr(self, attr):
                delattr(self, attr)
        self.n_neighbors = int(n_neighbors)
        self.n_components = int(n_components)
        self.n_epochs = None if n_epochs is None else int(n_epochs)
        self.metric, self.metric_kwds, self._metric_p = _metric_config(metric, metric_kwds)
        self.learning_rate = float(learning_rate)
        self.min_dist = float(min_dist)
        self.spread = float(spread)
        self.local_connectivity = float(local_connectivity)
        self.set_op_mix_ratio = float(set_op_mix_ratio)
        self.repulsion_strength = float(repulsion_strength)
        self.negative_sample_rate = int(negative_sample_rate)
        self.random_seed = int(random_seed)
        self.init = str(init)
        self.target_metric = _target_metric(target_metric)
        weight = float(target_weight)
        if not np.isfinite(weight) or weight < 0.0 or weight > 1.0:
            raise ValueError("target_weight must be finite and in [0, 1]")
        self.target_weight = weight
        if target_n_neighbors is not None and int(target_n_neighbors) < 1:
            raise ValueError("target_n_neighbors must be >= 1 when provided")
        self.target_n_neighbors = None if target_n_neighbors is None else int(target_n_neighbors)
        mode, use_approx, threshold = _ann_mode(ann_mode, use_approximate_knn, approx_knn_threshold)
        self.ann_mode = mode
        self.use_approximate_knn = bool(use_approx)
        self.approx_knn_candidates = int(approx_knn_candidates)
        self.approx_knn_iters = int(approx_knn_iters)
        self.approx_knn_threshold = int(threshold)
        self.densmap = bool(densmap)
        self.dens_lambda, self.dens_frac, self.dens_var_shift = _dens_params(
            dens_lambda, dens_frac, dens_var_shift
        )
        self.output_dens = bool(output_dens)
        self.knn_backend = str(knn_backend)
        if transform_mode not in _TRANSFORM_MODES:
            raise ValueError(f"transform_mode must be one of {_TRANSFORM_MODES}")
        self.transform_mode = str(transform_mode)
        self.surrogate_kwds = surrogate_kwds
        self._core = UmapCore(
            n_neighbors=self.n_neighbors,
            n_components=self.n_components,
            n_epochs=self.n_epochs,
            metric=self.metric,
            metric_p=self._metric_p,
            learning_rate=self.learning_rate,
            min_dist=self.min_dist,
            spread=self.spread,
            local_connectivity=self.local_connectivity,
            set_op_mix_ratio=self.set_op_mix_ratio,
            repulsion_strength=self.repulsion_strength,
            negative_sample_rate=self.negative_sample_rate,
            random_seed=self.random_seed,
            init=self.init,
            use_approximate_knn=self.use_approximate_knn,
            approx_knn_candidates=self.approx_knn_candidates,
            approx_knn_iters=self.approx_knn_iters,
            approx_knn_threshold=self.approx_knn_threshold,
            densmap=self.densmap,
            dens_lambda=self.dens_lambda,
            dens_frac=self.dens_frac,
            dens_var_shift=self.dens_var_shift,
            output_dens=self.output_dens,
            knn_backend=self.knn_backend,
        )

    # ------------------------------------------------------------ sklearn
    def get_params(self, deep: bool = True) -> dict[str, Any]:
        """Return constructor parameters for sklearn-compatible cloning."""
        return {name: getattr(self, name) for name in _PARAM_NAMES}

    def set_params(self, **params: Any) -> "Umap":
        """Set constructor parameters and rebuild the engine handle."""
        if not params:
            return self
        for key in params:
            if key not in _PARAM_NAMES:
                raise ValueError(f"Invalid parameter '{key}' for estimator Umap")
        current = self.get_params(deep=False)
        current.update(params)
        self.__init__(**current)
        return self

    def _set_fitted(self, embedding: np.ndarray, n_features: int, n_samples: int) -> None:
        self.embedding_ = embedding
        self.n_features_in_ = int(n_features)
        self.n_samples_fit_ = int(n_samples)
        self._sync_density_attributes()
        if self.transform_mode == "surrogate":
            self.fit_surrogate(**(self.surrogate_kwds or {}))

    def _sync_density_attributes(self) -> None:
        """radii_original_ / radii_embedding_ (and their rad_* aliases) after an
        output_dens fit, as the reference's facade keeps them (_api.py:530-541)."""
        radii_original = self._core.radii_original
        radii_embedding = self._core.radii_embedding
        if not self.output_dens or radii_original is None or radii_embedding is None:
            for attr in ("radii_original_", "radii_embedding_", "rad_orig_", "rad_emb_"):
                if hasattr(self, attr):
                    delattr(self, attr)
            return
        self.radii_original_ = radii_original
        self.radii_embedding_ = radii_embedding
        self.rad_orig_ = radii_original
        self.rad_emb_ = radii_embedding

    def fit_surrogate(self, **options: Any) -> dict[str, Any]:
        """Train the learned transform surrogate of the fitted model and
        return its training / held-out summary (also kept as
        ``surrogate_info_``)."""
        self.surrogate_info_ = self._core.fit_surrogate(**options)
        return self.surrogate_info_

    def _check_sparse_options(self, y: Any) -> None:
        if self.densmap or self.output_dens:
            raise ValueError("densmap and output_dens currently support dense input only")
        if self.target_metric == "categorical" and y is not None:
            raise ValueError("categorical supervised UMAP currently supports dense input only")

    # ---------------------------------------------------------------- fit
    def fit(self, data: Any, y: Any | None = None) -> "Umap":
        """Fit the model and return ``self``.

        Parameters
        ----------
        data:
            Converted to a C-contiguous ``float32`` matrix of shape
            ``(n_samples, n_features)``; a sparse matrix (csr, csc or coo) is
            fitted through its CSR form.
        y:
            Ignored unless ``target_metric="categorical"``.

        Returns
        -------
        Umap
            The fitted model.
        """
        csr = _maybe_as_csr_parts(data, "data")
        if csr is not None:
            self._check_sparse_options(y)
            indptr, indices, values, n_rows, n_cols = csr
            self._core.fit_sparse_csr(indptr, indices, values, n_cols)
            self._set_fitted(self._core.embedding, n_cols, n_rows)
            return self
        arr = _f32_matrix(data, "data")
        if self.target_metric == "categorical" and y is not None:
            labels = _as_labels(y, "y")
            self._core.fit_supervised(arr, labels, self.target_weight, self.target_n_neighbors)
            self._set_fitted(self._core.embedding, arr.shape[1], arr.shape[0])
            return self
        self._core.fit(arr)
        self._set_fitted(self._core.embedding, arr.shape[1], arr.shape[0])
        return self

    def fit_transform(
        self,
        data: Any,
        y: Any | None = None,
        *,
        out: np.ndarray | None = None,
    ) -> np.ndarray:
        """Fit the model and return the embedding of the training data.

        Parameters
        ----------
        data:
            Dense input, converted to ``float32`` of shape
            ``(n_samples, n_features)``, or a sparse matrix (csr, csc, coo).
        y:
            Ignored unless ``target_metric="categorical"``.
        out:
            Optional writable, C-contiguous buffer of dtype ``float32`` and
            shape ``(n_samples, n_components)``; filled in place and returned.

        Returns
        -------
        numpy.ndarray
            The embedding, dtype ``float32``, shape ``(n_samples, n_components)``.
        """
        csr = _maybe_as_csr_parts(data, "data")
        if csr is not None:
            if out is not None and self.output_dens:
                raise ValueError("out cannot be used when output_dens=True")
            self._check_sparse_options(y)
            indptr, indices, values, n_rows, n_cols = csr
            if out is None:
                emb = self._core.fit_transform_sparse_csr(indptr, indices, values, n_cols)
                self._set_fitted(emb, n_cols, n_rows)
                return emb
            buf = _out_buffer(out, (n_rows, self.n_components))
            self._core.fit_transform_sparse_csr_into(indptr, indices, values, n_cols, buf)
            self._set_fitted(buf, n_cols, n_rows)
            return buf
        arr = _f32_matrix(data, "data")
        if out is not None and self.output_dens:
            raise ValueError("out cannot be used when output_dens=True")
        if self.target_metric == "categorical" and y is not None:
            labels = _as_labels(y, "y")
            if out is None:
                emb = self._core.fit_transform_supervised(arr, labels, self.target_weight,
                                                          self.target_n_neighbors)
                self._set_fitted(emb, arr.shape[1], arr.shape[0])
                if self.output_dens:
                    return emb, self.radii_original_, self.radii_embedding_
                return emb
            buf = _out_buffer(out, (arr.shape[0], self.n_components))
            self._core.fit_transform_supervised_into(arr, labels, buf, self.target_weight,
                                                     self.target_n_neighbors)
            self._set_fitted(buf, arr.shape[1], arr.shape[0])
            return buf
        if out is None:
            emb = self._core.fit_transform(arr)
            self._set_fitted(emb, arr.shape[1], arr.shape[0])
            if self.output_dens:
                return emb, self.radii_original_, self.radii_embedding_
            return emb
        buf = _out_buffer(out, (arr.shape[0], self.n_components))
        self._core.fit_transform_into(arr, buf)
        self._set_fitted(buf, arr.shape[1], arr.shape[0])
        return buf

    def profile_fit_transform(self, data: Any) -> dict[str, Any]:
        """Fit dense input and return the embedding with a per-stage timing
        breakdown (same keys as the reference's FitTimingBreakdown)."""
        if _is_sparse(data):
            raise ValueError("profile_fit_transform currently supports dense input only")
        if self.target_metric is not None:
            raise ValueError("profile_fit_transform currently supports unsupervised input only")
        if self.densmap or self.output_dens:
            raise ValueError("profile_fit_transform currently supports standard UMAP only")
        arr = _f32_matrix(data, "data")
        result = self._core.profile_fit_transform(arr)
        self._set_fitted(result["embedding"], arr.shape[1], arr.shape[0])
        return result

    def fit_transform_with_knn(
        self,
        data: Any,
        knn_indices: Any,
        knn_dists: Any,
        *,
        knn_metric: str = "euclidean",
        validate_precomputed: bool = True,
        out: np.ndarray | None = None,
    ) -> np.ndarray:
        """Fit from a precomputed kNN graph and return the embedding.

        An advanced entry point for callers that already hold neighbour lists
        (from another index, or a cached run): the kNN stage is skipped and
        the given lists feed the fuzzy graph directly.

        Parameters
        ----------
        data:
            Dense training data ``(n_samples, n_features)``.
        knn_indices:
            Neighbour indices ``(n_samples, k)``, integer dtype, ``k >= n_neighbors``.
        knn_dists:
            Neighbour distances ``(n_samples, k)``, non-decreasing per row.
        knn_metric:
            Metric of the precomputed graph; must match the model metric.
        validate_precomputed:
            Check that every distance is finite and non-negative first.
        out:
            Optional writable ``float32`` buffer ``(n_samples, n_components)``.

        Returns
        -------
        numpy.ndarray
            The embedding.
        """
        arr = _f32_matrix(data, "data")
        idx = _i64_matrix(knn_indices, "knn_indices")
        dist = _f32_matrix(knn_dists, "knn_dists")
        if out is None:
            emb = self._core.fit_transform_with_knn(arr, idx, dist, knn_metric, validate_precomputed)
        else:
            emb = _out_buffer(out, (arr.shape[0], self.n_components))
            self._core.fit_transform_with_knn_into(arr, idx, dist, emb, knn_metric, validate_precomputed)
        self._set_fitted(emb, arr.shape[1], arr.shape[0])
        return emb

    def knn_diagnostics(self, data: Any) -> dict[str, Any]:
        """Recall of NN-descent against exact neighbours on ``data``."""
        arr = _f32_matrix(data, "data")
        diag = self._core.knn_recall_diagnostics(arr)
        self.knn_diagnostics_ = diag
        return diag

    # ---------------------------------------------------------- transform
    def transform(self, query: Any, *, out: np.ndarray | None = None,
                  method: str | None = None) -> np.ndarray:
        """Place new samples in the fitted embedding.

        Parameters
        ----------
        query:
            Dense input ``(n_samples, n_features)``, or a sparse matrix for a
            model fitted on sparse input.
        out:
            Optional writable ``float32`` buffer ``(n_samples, n_components)``.
        method:
            ``plain`` | ``surrogate``; default ``transform_mode``.  With the
            surrogate, ``transform_fallback_`` records which rows the gate
            sent to the plain transform.

        Returns
        -------
        numpy.ndarray
            The projected embedding.
        """
        csr = _maybe_as_csr_parts(query, "query")
        if csr is not None:
            indptr, indices, values, n_rows, n_cols = csr
            if out is None:
                return self._core.transform_sparse_csr(indptr, indices, values, n_cols)
            buf = _out_buffer(out, (n_rows, self.n_components))
            self._core.transform_sparse_csr_into(indptr, indices, values, n_cols, buf)
            return buf
        arr = _f32_matrix(query, "query")
        method = self.transform_mode if method is None else method
        if method not in _TRANSFORM_MODES:
            raise ValueError(f"method must be one of {_TRANSFORM_MODES}")
        if method == "surrogate":
            emb, flags = self._core.transform_surrogate(arr, use_fallback=True)
            self.transform_fallback_ = flags
            if out is None:
                return emb
            buf = _out_buffer(out, (arr.shape[0], self.n_components))
            buf[...] = emb
            return buf
        if out is None:
            return self._core.transform(arr)
        buf = _out_buffer(out, (arr.shape[0], self.n_components))
        self._core.transform_into(arr, buf)
        return buf

    def inverse_transform(self, embedded_query: Any, *, out: np.ndarray | None = None) -> np.ndarray:
        """Map embedded samples back to the feature space (_api.py:838-873).

        Parameters
        ----------
        embedded_query:
            Dense embedding of shape ``(n_samples, n_components)``, converted
            to ``float32``.
        out:
            Optional writable ``float32`` buffer of shape
            ``(n_samples, n_features)``; the model must be fit first.

        Returns
        -------
        numpy.ndarray
            The reconstructed samples, shape ``(n_samples, n_features)``.
        """
        arr = _f32_matrix(embedded_query, "embedded_query")
        if out is None:
            return self._core.inverse_transform(arr)
        n_features = self._core.n_features
        if n_features is None:
            raise RuntimeError("model must be fit before inverse_transform(out=...)")
        buf = _out_buffer(out, (arr.shape[0], n_features))
        self._core.inverse_transform_into(arr, buf)
        return buf


class ParametricUmap:
    """Placeholder for the reference's teacher-distilled MLP estimator, which
    the B200 engine does not provide."""

    def __init__(self, *args: Any, **kwargs: Any) -> None:
        ParametricUmapCore()


class AlignedUmap:
    """Placeholder for the reference's aligned multi-slice estimator, which
    the B200 engine does not provide."""

    def __init__(self, *args: Any, **kwargs: Any) -> None:
        AlignedUmapCore()


def fit_transform(data: Any, y: Any | None = None, **kwargs: Any) -> np.ndarray:
    """Embed a dataset in one call (no model state is kept).

    Parameters
    ----------
    data:
        Dense input accepted by ``Umap.fit_transform``.
    y:
        Ignored unless ``target_metric="categorical"``.
    **kwargs:
        Hyperparameters forwarded to ``Umap(...)``.

    Returns
    -------
    numpy.ndarray
        Embedding of shape ``(n_samples, n_components)``, dtype ``float32``.
    """
    model = Umap(**kwargs)
    if y is None and model.target_metric is None and not model.densmap and not model.output_dens:
        csr = _maybe_as_csr_parts(data, "data")
        if csr is not None:
            indptr, indices, values, _, n_cols = csr
            return model._core.fit_transform_sparse_csr_stateless(indptr, indices, values, n_cols)
        return model._core.fit_transform_stateless(_f32_matrix(data, "data"))
    return model.fit_transform(data, y=y)
