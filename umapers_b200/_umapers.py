"""``UmapCore``: the engine class behind ``Umap``, over the C ABI.

Mirrors the PyO3 class ``umapers._umapers.UmapCore`` (umap_rs/src/lib.rs:
540-1320): the same constructor keywords and defaults, the same methods and
getters, and the same error mapping (NotFitted and device failures raise
RuntimeError, everything else ValueError).  Every compute call goes through
libumapb200.so; ctypes releases the GIL for the duration of the call, as the
reference's ``py.allow_threads`` does.  One keyword is added: ``knn_backend``
("auto" | "tensor" | "plain") selects how exact kNN tiles are computed.
"""
from __future__ import annotations

import ctypes
from typing import Any

import numpy as np

from . import _lib

__version__ = "1.1.4"


def _parse_metric(metric: str, metric_p: float | None) -> tuple[int, float]:
    """parse_metric (umap_rs/src/lib.rs:22-48)."""
    name = str(metric).lower()
    aliases = {"l2": "euclidean", "l1": "manhattan", "linfinity": "chebyshev",
               "linf": "chebyshev", "bray_curtis": "braycurtis"}
    name = aliases.get(name, name)
    if name not in _lib.METRICS:
        raise ValueError(
            f"unsupported metric '{metric}', expected "
            "euclidean|manhattan|cosine|chebyshev|minkowski|correlation|canberra|braycurtis"
        )
    p = 0.0
    if name == "minkowski":
        if metric_p is None:
            raise ValueError("metric='minkowski' requires metric_kwds={'p': ...}")
        p = float(metric_p)
        if not np.isfinite(p) or p <= 0.0:
            raise ValueError("metric_kwds['p'] must be finite and > 0 for minkowski")
    return _lib.METRICS[name], p


def _parse_init(init: str) -> int:
    """parse_init (umap_rs/src/lib.rs:127-135)."""
    name = str(init).lower()
    if name == "random":
        return 0
    if name == "spectral":
        return 1
    raise ValueError(f"unsupported init '{init}', expected random|spectral")


def _usize(value: Any, name: str) -> int:
    v = int(value)
    if v < 0:
        raise OverflowError(f"can't convert negative int to unsigned ({name})")
    return v


def _matrix(x: Any, name: str) -> np.ndarray:
    """A C-contiguous float32 2-D view of x, rejecting zero columns as the
    PyO3 binding does (ensure_nonzero_columns, umap_rs/src/lib.rs:166-178)."""
    arr = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    if arr.ndim != 2:
        raise ValueError(f"{name} must be a 2D array, got ndim={arr.ndim}")
    if arr.shape[1] == 0:
        raise ValueError(f"{name} must have at least one column")
    return arr


def _check_out(out: np.ndarray, shape: tuple[int, int]) -> None:
    """copy_dense_into_out shape check (umap_rs/src/lib.rs:511-538)."""
    if tuple(out.shape) != tuple(shape):
        raise ValueError(
            f"output buffer shape mismatch: expected ({shape[0]}, {shape[1]}), "
            f"got ({out.shape[0]}, {out.shape[1]})"
        )
    if out.dtype != np.float32 or not out.flags.c_contiguous or not out.flags.writeable:
        raise ValueError("output buffer must be a writeable C-contiguous float32 array")


def _nonneg_i64(x: Any, name: str) -> np.ndarray:
    """i64_slice_to_usize_vec (umap_rs/src/lib.rs:242-260)."""
    arr = np.ascontiguousarray(np.asarray(x, dtype=np.int64))
    if arr.ndim != 1:
        raise ValueError(f"{name} must be a 1D array")
    if arr.size and int(arr.min()) < 0:
        raise ValueError(f"{name} must contain non-negative integers")
    return arr


def _csr_arrays(indptr: Any, indices: Any, data: Any, n_cols: int):
    """sparse_csr_from_py (umap_rs/src/lib.rs:337-351) and the length checks
    of SparseCsrMatrix::new (rust_umap/src/sparse.rs:20-56); the per-row
    checks run in the engine."""
    ip = _nonneg_i64(indptr, "indptr")
    ix = _nonneg_i64(indices, "indices")
    dv = np.ascontiguousarray(np.asarray(data, dtype=np.float32))
    if dv.ndim != 1:
        raise ValueError("data must be a 1D array")
    if ip.shape[0] == 0:
        raise ValueError("indptr cannot be empty")
    n_rows = ip.shape[0] - 1
    if int(n_cols) < 1:
        raise ValueError("invalid parameter: csr n_cols must be >= 1")
    if ip[0] != 0:
        raise ValueError("invalid parameter: csr indptr must start from 0")
    if ix.shape[0] != dv.shape[0]:
        raise ValueError("invalid parameter: csr indices/data lengths must match")
    if ip[n_rows] != ix.shape[0]:
        raise ValueError(f"invalid parameter: csr indptr last value ({int(ip[n_rows])}) must "
                         f"equal nnz ({ix.shape[0]})")
    return ip, ix, dv, n_rows, int(n_cols)


class UmapCore:
    """Engine handle with the ``UmapCore`` surface of the reference binding."""

    def __init__(
        self,
        n_neighbors: int = 15,
        n_components: int = 2,
        n_epochs: int | None = None,
        metric: str = "euclidean",
        metric_p: float | None = None,
        learning_rate: float = 1.0,
        min_dist: float = 0.1,
        spread: float = 1.0,
        local_connectivity: float = 1.0,
        set_op_mix_ratio: float = 1.0,
        repulsion_strength: float = 1.0,
        negative_sample_rate: int = 5,
        random_seed: int = 42,
        init: str = "spectral",
        use_approximate_knn: bool = True,
        approx_knn_candidates: int = 50,
        approx_knn_iters: int = 14,
        approx_knn_threshold: int = 4096,
        densmap: bool = False,
        dens_lambda: float = 2.0,
        dens_frac: float = 0.3,
        dens_var_shift: float = 0.1,
        output_dens: bool = False,
        knn_backend: str = "auto",
    ) -> None:
        lib = _lib.load()
        metric_id, p = _parse_metric(metric, metric_p)
        params = _lib.Params()
        lib.umapb_params_default(ctypes.byref(params))
        params.n_neighbors = _usize(n_neighbors, "n_neighbors")
        params.n_components = _usize(n_components, "n_components")
        params.n_epochs = -1 if n_epochs is None else _usize(n_epochs, "n_epochs")
        params.metric = metric_id
        params.metric_p = p
        params.learning_rate = float(learning_rate)
        params.min_dist = float(min_dist)
        params.spread = float(spread)
        params.local_connectivity = float(local_connectivity)
        params.set_op_mix_ratio = float(set_op_mix_ratio)
        params.repulsion_strength = float(repulsion_strength)
        params.negative_sample_rate = _usize(negative_sample_rate, "negative_sample_rate")
        params.random_seed = int(random_seed) & 0xFFFFFFFFFFFFFFFF
        params.init = _parse_init(init)
        params.use_approximate_knn = int(bool(use_approximate_knn))
        params.approx_knn_candidates = _usize(approx_knn_candidates, "approx_knn_candidates")
        params.approx_knn_iters = _usize(approx_knn_iters, "approx_knn_iters")
        params.approx_knn_threshold = _usize(approx_knn_threshold, "approx_knn_threshold")
        params.densmap = int(bool(densmap))
        params.dens_lambda = float(dens_lambda)
        params.dens_frac = float(dens_frac)
        params.dens_var_shift = float(dens_var_shift)
        params.output_dens = int(bool(output_dens))
        if knn_backend not in _lib.KNN_BACKENDS:
            raise ValueError(f"unsupported knn_backend '{knn_backend}', expected auto|tensor|plain")
        params.knn_backend = _lib.KNN_BACKENDS[knn_backend]
        self._params = params
        self._metric_id = metric_id
        handle = ctypes.c_void_p()
        _lib.check(lib.umapb_create(ctypes.byref(params), ctypes.byref(handle)))
        self._handle = handle
        self._lib = lib

    def __del__(self) -> None:
        handle = getattr(self, "_handle", None)
        if handle is not None and handle.value:
            self._lib.umapb_destroy(handle)
            self._handle = None

    # ------------------------------------------------------------- fitting
    def fit(self, data: Any) -> None:
        arr = _matrix(data, "data")
        _lib.check(self._lib.umapb_fit(self._handle, _lib.ptr(arr), arr.shape[0], arr.shape[1]))

    def fit_transform(self, data: Any) -> np.ndarray:
        arr = _matrix(data, "data")
        out = np.empty((arr.shape[0], self.n_components), dtype=np.float32)
        _lib.check(
            self._lib.umapb_fit_transform(
                self._handle, _lib.ptr(arr), arr.shape[0], arr.shape[1], _lib.ptr(out)
            )
        )
        return out

    def fit_transform_into(self, data: Any, out: np.ndarray) -> None:
        arr = _matrix(data, "data")
        _check_out(out, (arr.shape[0], self.n_components))
        _lib.check(
            self._lib.umapb_fit_transform(
                self._handle, _lib.ptr(arr), arr.shape[0], arr.shape[1], _lib.ptr(out)
            )
        )

    # ------------------------------------------- categorical supervision
    @staticmethod
    def _target(y: Any, target_weight: float, target_n_neighbors: int | None):
        """Labels as int64 (PyReadonlyArray1<i64>), the weight as f32 and
        target_n_neighbors as Option<usize> (-1 for none) of the reference's
        supervised_target_from_py (umap_rs/src/lib.rs:324-335)."""
        labels = np.ascontiguousarray(y, dtype=np.int64)
        if labels.ndim != 1:
            raise ValueError(f"y must be a 1D label array, got ndim={labels.ndim}")
        if target_n_neighbors is None:
            tnn = -1
        else:
            tnn = int(target_n_neighbors)
            if tnn < 0:
                raise OverflowError("can't convert negative int to unsigned")
        return labels, float(target_weight), tnn

    def fit_supervised(self, data: Any, y: Any, target_weight: float,
                       target_n_neighbors: int | None = None) -> None:
        """UmapCore.fit_supervised (umap_rs/src/lib.rs:647-673)."""
        arr = _matrix(data, "data")
        labels, weight, tnn = self._target(y, target_weight, target_n_neighbors)
        _lib.check(
            self._lib.umapb_fit_supervised(self._handle, _lib.ptr(arr), arr.shape[0], arr.shape[1],
                                           _lib.ptr(labels), labels.shape[0], weight, tnn)
        )

    def fit_transform_supervised(self, data: Any, y: Any, target_weight: float,
                                 target_n_neighbors: int | None = None) -> np.ndarray:
        """UmapCore.fit_transform_supervised (umap_rs/src/lib.rs:746-779)."""
        arr = _matrix(data, "data")
        labels, weight, tnn = self._target(y, target_weight, target_n_neighbors)
        out = np.empty((arr.shape[0], self.n_components), dtype=np.float32)
        _lib.check(
            self._lib.umapb_fit_transform_supervised(
                self._handle, _lib.ptr(arr), arr.shape[0], arr.shape[1], _lib.ptr(labels),
                labels.shape[0], weight, tnn, _lib.ptr(out)
            )
        )
        return out

    def fit_transform_supervised_into(self, data: Any, y: Any, out: np.ndarray,
                                      target_weight: float,
                                      target_n_neighbors: int | None = None) -> None:
        """UmapCore.fit_transform_supervised_into (umap_rs/src/lib.rs:835-868)."""
        arr = _matrix(data, "data")
        labels, weight, tnn = self._target(y, target_weight, target_n_neighbors)
        _check_out(out, (arr.shape[0], self.n_components))
        _lib.check(
            self._lib.umapb_fit_transform_supervised(
                self._handle, _lib.ptr(arr), arr.shape[0], arr.shape[1], _lib.ptr(labels),
                labels.shape[0], weight, tnn, _lib.ptr(out)
            )
        )

    def fit_transform_stateless(self, data: Any) -> np.ndarray:
        arr = _matrix(data, "data")
        out = np.empty((arr.shape[0], self.n_components), dtype=np.float32)
        _lib.check(
            self._lib.umapb_fit_transform_stateless(
                ctypes.byref(self._params), _lib.ptr(arr), arr.shape[0], arr.shape[1],
                _lib.ptr(out),
            )
        )
        return out

    def profile_fit_transform(self, data: Any) -> dict[str, Any]:
        """Same dict schema as the reference (umap_rs/src/lib.rs:88-125), with
        B200 counters added under their own keys."""
        arr = _matrix(data, "data")
        out = np.empty((arr.shape[0], self.n_components), dtype=np.float32)
        timings = _lib.Timings()
        info = _lib.FitInfo()
        _lib.check(
            self._lib.umapb_profile_fit_transform(
                self._handle, _lib.ptr(arr), arr.shape[0], arr.shape[1], _lib.ptr(out),
                ctypes.byref(timings), ctypes.byref(info),
            )
        )
        backend = {-1: "nndescent", 0: "auto", 1: "tensor", 2: "plain"}.get(
            info.knn_backend_used, "unknown"
        )
        return {
            "embedding": out,
            "timings": {name: float(getattr(timings, name)) for name in _lib.TIMING_FIELDS},
            "used_approximate_knn": bool(info.used_approximate_knn),
            "n_samples": int(info.n_samples),
            "n_features": int(info.n_features),
            "n_epochs": int(info.n_epochs),
            "n_edges": int(info.n_edges),
            "knn_backend": backend,
            "knn_fallback_rows": int(info.knn_fallback_rows),
            "knn_second_pass_rows": int(info.knn_second_pass_rows),
            "knn_kernel_sec": float(info.knn_kernel_sec),
            "n_graph_components": int(info.n_components_graph),
            "sgd_edge_samples": float(info.sgd_edge_samples),
        }

    def _with_knn(self, data, knn_indices, knn_dists, out, knn_metric, validate_precomputed):
        arr = _matrix(data, "data")
        metric_id, _ = _parse_metric(knn_metric, None if knn_metric != "minkowski" else 1.0)
        idx = np.ascontiguousarray(np.asarray(knn_indices, dtype=np.int64))
        dist = np.ascontiguousarray(np.asarray(knn_dists, dtype=np.float32))
        if idx.ndim != 2:
            raise ValueError(f"knn_indices must be a 2D array, got ndim={idx.ndim}")
        if dist.ndim != 2:
            raise ValueError(f"knn_dists must be a 2D array, got ndim={dist.ndim}")
        _lib.check(
            self._lib.umapb_fit_transform_with_knn(
                self._handle, _lib.ptr(arr), arr.shape[0], arr.shape[1], _lib.ptr(idx),
                idx.shape[0], idx.shape[1], _lib.ptr(dist), dist.shape[0], dist.shape[1],
                metric_id, int(bool(validate_precomputed)), _lib.ptr(out),
            )
        )

    def fit_transform_with_knn(
        self,
        data: Any,
        knn_indices: Any,
        knn_dists: Any,
        knn_metric: str = "euclidean",
        validate_precomputed: bool = True,
    ) -> np.ndarray:
        n_rows = np.shape(data)[0]
        out = np.empty((n_rows, self.n_components), dtype=np.float32)
        self._with_knn(data, knn_indices, knn_dists, out, knn_metric, validate_precomputed)
        return out

    def fit_transform_with_knn_into(
        self,
        data: Any,
        knn_indices: Any,
        knn_dists: Any,
        out: np.ndarray,
        knn_metric: str = "euclidean",
        validate_precomputed: bool = True,
    ) -> None:
        _check_out(out, (np.shape(data)[0], self.n_components))
        self._with_knn(data, knn_indices, knn_dists, out, knn_metric, validate_precomputed)

    # ----------------------------------------------------------- transform
    def transform(self, query: Any) -> np.ndarray:
        arr = _matrix(query, "query")
        out = np.empty((arr.shape[0], self.n_components), dtype=np.float32)
        _lib.check(
            self._lib.umapb_transform(
                self._handle, _lib.ptr(arr), arr.shape[0], arr.shape[1], _lib.ptr(out)
            )
        )
        return out

    def transform_into(self, query: Any, out: np.ndarray) -> None:
        arr = _matrix(query, "query")
        _check_out(out, (arr.shape[0], self.n_components))
        _lib.check(
            self._lib.umapb_transform(
                self._handle, _lib.ptr(arr), arr.shape[0], arr.shape[1], _lib.ptr(out)
            )
        )

    # --------------------------------------------------------- CSR input
    # fit_sparse_csr / fit_transform_sparse_csr[_into|_stateless] /
    # transform_sparse_csr[_into] (umap_rs/src/lib.rs:674-686, 869-915,
    # 1198-1227).
    def fit_sparse_csr(self, indptr: Any, indices: Any, data: Any, n_cols: int) -> None:
        ip, ix, dv, n, d = _csr_arrays(indptr, indices, data, n_cols)
        _lib.check(self._lib.umapb_fit_csr(self._handle, _lib.ptr(ip), _lib.ptr(ix),
                                           _lib.ptr(dv), n, d))

    def fit_transform_sparse_csr(self, indptr: Any, indices: Any, data: Any,
                                 n_cols: int) -> np.ndarray:
        ip, ix, dv, n, d = _csr_arrays(indptr, indices, data, n_cols)
        out = np.empty((n, self.n_components), dtype=np.float32)
        _lib.check(self._lib.umapb_fit_transform_csr(self._handle, _lib.ptr(ip), _lib.ptr(ix),
                                                     _lib.ptr(dv), n, d, _lib.ptr(out)))
        return out

    def fit_transform_sparse_csr_into(self, indptr: Any, indices: Any, data: Any, n_cols: int,
                                      out: np.ndarray) -> None:
        ip, ix, dv, n, d = _csr_arrays(indptr, indices, data, n_cols)
        _check_out(out, (n, self.n_components))
        _lib.check(self._lib.umapb_fit_transform_csr(self._handle, _lib.ptr(ip), _lib.ptr(ix),
                                                     _lib.ptr(dv), n, d, _lib.ptr(out)))

    def fit_transform_sparse_csr_stateless(self, indptr: Any, indices: Any, data: Any,
                                           n_cols: int) -> np.ndarray:
        ip, ix, dv, n, d = _csr_arrays(indptr, indices, data, n_cols)
        out = np.empty((n, self.n_components), dtype=np.float32)
        _lib.check(self._lib.umapb_fit_transform_csr_stateless(
            ctypes.byref(self._params), _lib.ptr(ip), _lib.ptr(ix), _lib.ptr(dv), n, d,
            _lib.ptr(out)))
        return out

    def transform_sparse_csr(self, indptr: Any, indices: Any, data: Any,
                             n_cols: int) -> np.ndarray:
        ip, ix, dv, n, d = _csr_arrays(indptr, indices, data, n_cols)
        out = np.empty((n, self.n_components), dtype=np.float32)
        _lib.check(self._lib.umapb_transform_csr(self._handle, _lib.ptr(ip), _lib.ptr(ix),
                                                 _lib.ptr(dv), n, d, _lib.ptr(out)))
        return out

    def transform_sparse_csr_into(self, indptr: Any, indices: Any, data: Any, n_cols: int,
                                  out: np.ndarray) -> None:
        ip, ix, dv, n, d = _csr_arrays(indptr, indices, data, n_cols)
        _check_out(out, (n, self.n_components))
        _lib.check(self._lib.umapb_transform_csr(self._handle, _lib.ptr(ip), _lib.ptr(ix),
                                                 _lib.ptr(dv), n, d, _lib.ptr(out)))

    # ------------------------------------------------- learned surrogate
    # No reference counterpart (the reference's ParametricUmapCore is a
    # separate estimator): a BF16 MLP trained on this model's fit maps rows
    # straight to the embedding; rows its gate rejects take the plain path.
    def fit_surrogate(self, **options: Any) -> dict[str, Any]:
        """Train the transform surrogate of the fitted model.  Keyword options
        are the fields of ``umapb_surrogate_params`` (hidden, epochs,
        batch_size, learning_rate, mse_weight, edge_loss_weight, negatives,
        holdout_fraction, n_anchors, fallback_radius, max_cell_failure, seed).
        Returns the training and calibration summary."""
        prm = _lib.SurrogateParams()
        self._lib.umapb_surrogate_params_default(ctypes.byref(prm))
        names = {f[0] for f in _lib.SurrogateParams._fields_}
        for key, value in options.items():
            if key not in names:
                raise ValueError(f"unknown surrogate option: {key}")
            setattr(prm, key, value)
        info = _lib.SurrogateInfo()
        _lib.check(self._lib.umapb_surrogate_fit(self._handle, ctypes.byref(prm),
                                                 ctypes.byref(info)))
        return {name: getattr(info, name) for name, _ in _lib.SURROGATE_INFO_FIELDS}

    @property
    def surrogate_ready(self) -> bool:
        return bool(self._lib.umapb_surrogate_ready(self._handle))

    def transform_surrogate(self, query: Any, use_fallback: bool = True
                            ) -> tuple[np.ndarray, np.ndarray]:
        """Embedding of new rows through the surrogate and, per row, whether
        the gate sent it to the plain transform (recomputed there when
        ``use_fallback``)."""
        arr = _matrix(query, "query")
        out = np.empty((arr.shape[0], self.n_components), dtype=np.float32)
        flags = np.empty(arr.shape[0], dtype=np.uint8)
        n_fb = ctypes.c_int64(0)
        _lib.check(self._lib.umapb_surrogate_transform(
            self._handle, _lib.ptr(arr), arr.shape[0], arr.shape[1], 1 if use_fallback else 0,
            _lib.ptr(out), _lib.ptr(flags), ctypes.byref(n_fb)))
        return out, flags.astype(bool)

    def surrogate_loss_history(self) -> np.ndarray:
        """Mean training loss of each epoch of the last fit_surrogate."""
        buf = np.empty(4096, dtype=np.float64)
        n = ctypes.c_int64(0)
        _lib.check(self._lib.umapb_surrogate_loss_history(self._handle, _lib.ptr(buf), buf.size,
                                                          ctypes.byref(n)))
        return buf[: n.value].copy()

    def inverse_transform(self, embedded_query: Any) -> np.ndarray:
        """UmapCore.inverse_transform (umap_rs/src/lib.rs:1229-1252): rows of
        the embedding mapped back to the feature space."""
        arr = _matrix(embedded_query, "embedded_query")
        out = np.empty((arr.shape[0], self.n_features or 0), dtype=np.float32)
        _lib.check(
            self._lib.umapb_inverse_transform(
                self._handle, _lib.ptr(arr), arr.shape[0], arr.shape[1], _lib.ptr(out)
            )
        )
        return out

    def inverse_transform_into(self, embedded_query: Any, out: np.ndarray) -> None:
        """UmapCore.inverse_transform_into (umap_rs/src/lib.rs:1254-1290)."""
        arr = _matrix(embedded_query, "embedded_query")
        _check_out(out, (arr.shape[0], self.n_features or 0))
        _lib.check(
            self._lib.umapb_inverse_transform(
                self._handle, _lib.ptr(arr), arr.shape[0], arr.shape[1], _lib.ptr(out)
            )
        )

    # --------------------------------------------------------- diagnostics
    def knn_recall_diagnostics(self, data: Any) -> dict[str, Any]:
        """approximate_knn_recall_diagnostics_dense (rust_umap/src/lib.rs:2333-2437):
        exact and NN-descent kNN on the GPU, recall per row excluding self."""
        arr = _matrix(data, "data")
        n, d = arr.shape
        if n == 0:
            raise ValueError("input data is empty")
        if n < 2:
            raise ValueError("need at least two samples")
        p = self._params
        if p.n_neighbors < 2:
            raise ValueError("invalid parameter: n_neighbors must be >= 2")
        if p.n_neighbors >= n:
            raise ValueError(
                f"invalid parameter: n_neighbors ({p.n_neighbors}) must be smaller than "
                f"number of samples ({n})"
            )
        k = min(p.n_neighbors, n)
        pool = min(max(p.approx_knn_candidates, k), n - 1)
        seed = (p.random_seed ^ 0xC0FEFEED1234ABCD) & 0xFFFFFFFFFFFFFFFF
        ex_i = np.empty((n, k), np.int64)
        ex_d = np.empty((n, k), np.float32)
        _lib.check(self._lib.umapb_knn_exact(_lib.ptr(arr), n, d, k, p.metric, p.knn_backend,
                                             _lib.ptr(ex_i), _lib.ptr(ex_d), None))
        ap_i = np.empty((n, k), np.int64)
        ap_d = np.empty((n, k), np.float32)
        _lib.check(self._lib.umapb_nndescent(_lib.ptr(arr), n, d, k, p.metric,
                                             p.approx_knn_candidates, p.approx_knn_iters, seed,
                                             _lib.ptr(ap_i), _lib.ptr(ap_d), None, None, None))
        per_row = np.empty(n, np.float32)
        rows = np.arange(n)
        for r in range(n):
            exact = set(ex_i[r].tolist()) - {r}
            if not exact:
                per_row[r] = 1.0
                continue
            got = sum(1 for j in ap_i[r].tolist() if j != r and j in exact)
            per_row[r] = np.float32(got) / np.float32(len(exact))
        del rows
        worst = max(1, -(-n // 10))
        srt = np.sort(per_row)
        metric_name = [k_ for k_, v in _lib.METRICS.items() if v == p.metric][0]
        return {
            "n_samples": n,
            "n_features": d,
            "n_neighbors": k,
            "metric": metric_name,
            "metric_p": float(p.metric_p) if metric_name == "minkowski" else None,
            "candidate_pool": pool,
            "n_iters": int(p.approx_knn_iters),
            "seed": seed,
            "mean_recall": float(per_row.mean()),
            "min_recall": float(per_row.min()),
            "worst_decile_recall": float(srt[:worst].mean()),
            "per_row_recall": per_row,
        }

    # ------------------------------------------------------------- getters
    @property
    def n_components(self) -> int:
        return int(self._lib.umapb_n_components(self._handle))

    @property
    def n_neighbors(self) -> int:
        return int(self._lib.umapb_n_neighbors(self._handle))

    @property
    def n_features(self) -> int | None:
        v = int(self._lib.umapb_n_features(self._handle))
        return None if v < 0 else v

    @property
    def embedding(self) -> np.ndarray | None:
        n = int(self._lib.umapb_n_samples(self._handle))
        if n < 0:
            return None
        out = np.empty((n, self.n_components), dtype=np.float32)
        _lib.check(self._lib.umapb_get_embedding(self._handle, _lib.ptr(out), n, self.n_components))
        return out

    def _radii(self, which: int) -> np.ndarray | None:
        if not self._lib.umapb_has_radii(self._handle):
            return None
        n = self._lib.umapb_n_samples(self._handle)
        out = np.empty(n, dtype=np.float32)
        ptrs = [None, None]
        ptrs[which] = _lib.ptr(out)
        _lib.check(self._lib.umapb_get_radii(self._handle, ptrs[0], ptrs[1], n))
        return out

    @property
    def radii_original(self) -> np.ndarray | None:
        """Mean log neighbour radius of each fitted row in the input space
        (densmap / output_dens fits only)."""
        return self._radii(0)

    @property
    def radii_embedding(self) -> np.ndarray | None:
        """The same radius measured in the embedding."""
        return self._radii(1)

    @property
    def ab_params(self) -> tuple[float, float] | None:
        a = ctypes.c_float()
        b = ctypes.c_float()
        if self._lib.umapb_get_ab(self._handle, ctypes.byref(a), ctypes.byref(b)) != _lib.OK:
            return None
        return float(a.value), float(b.value)


class ParametricUmapCore:  # pragma: no cover - surface placeholder
    def __init__(self, *args: Any, **kwargs: Any) -> None:
        raise ValueError("ParametricUmap is not provided by the B200 engine")


class AlignedUmapCore:  # pragma: no cover - surface placeholder
    def __init__(self, *args: Any, **kwargs: Any) -> None:
        raise ValueError("AlignedUmap is not provided by the B200 engine")
