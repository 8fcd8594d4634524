"""Host-side behaviour of the umapers surface (no GPU): parameters,
normalisation and the reference's validation errors, which all fire before
any device work.  Mirrors umap_rs/tests/test_binding.py and the error
contracts of rust_umap/src/lib.rs tests."""
import inspect

import numpy as np
import pytest

import umapers
import umapers._api as api
from umapers import Umap, fit_transform
from umapers._umapers import UmapCore
from umapers_b200 import workloads


def test_public_api_has_docstrings():
    for obj in (Umap, Umap.__init__, Umap.fit, Umap.fit_transform, Umap.fit_transform_with_knn,
                Umap.transform, fit_transform):
        assert len(inspect.getdoc(obj) or "") > 40


def test_top_level_fit_transform_signature():
    sig = inspect.signature(fit_transform)
    assert list(sig.parameters)[:2] == ["data", "y"]


def test_get_params_returns_constructor_arguments():
    m = Umap(n_neighbors=9, metric="l2", ann_mode="exact", random_seed=3)
    p = m.get_params()
    assert p["n_neighbors"] == 9 and p["metric"] == "euclidean" and p["random_seed"] == 3
    assert p["use_approximate_knn"] is False and p["ann_mode"] == "exact"
    assert set(api._PARAM_NAMES) == set(p)


def test_set_params_rebuilds_and_clears_fitted_attributes():
    m = Umap()
    m.embedding_ = np.zeros((2, 2), np.float32)
    core = m._core
    m.set_params(n_neighbors=7)
    assert m.n_neighbors == 7 and m._core is not core and not hasattr(m, "embedding_")
    with pytest.raises(ValueError, match="Invalid parameter"):
        m.set_params(bogus=1)


def test_ann_mode_overrides_flags():
    assert Umap(ann_mode="approximate").approx_knn_threshold == 0
    assert Umap(ann_mode="approximate").use_approximate_knn is True
    assert Umap(ann_mode="exact", use_approximate_knn=True).use_approximate_knn is False
    with pytest.raises(ValueError, match="ann_mode"):
        Umap(ann_mode="fast")


def test_unsupported_metric_and_init_are_rejected():
    with pytest.raises(ValueError, match="unsupported metric"):
        Umap(metric="hamming")
    with pytest.raises(ValueError, match="unsupported init"):
        Umap(init="pca")
    with pytest.raises(ValueError, match="requires metric_kwds"):
        Umap(metric="minkowski")


def test_non_finite_input_is_rejected():
    # rust_umap/src/lib.rs:6662-6680
    x = workloads.reference_synthetic(32, 6)
    x[7, 3] = np.nan
    with pytest.raises(ValueError, match="non-finite value at row 7"):
        Umap(n_neighbors=8, n_epochs=20, init="random").fit_transform(x)


def test_non_finite_hyperparameter_is_rejected():
    # rust_umap/src/lib.rs:6683-6705
    x = workloads.reference_synthetic(32, 6)
    with pytest.raises(ValueError, match="learning_rate must be finite"):
        Umap(n_neighbors=8, learning_rate=float("inf")).fit_transform(x)


@pytest.mark.parametrize(
    "kwargs, msg",
    [
        (dict(n_neighbors=1), "n_neighbors must be >= 2"),
        (dict(n_neighbors=40), "must be smaller than number of samples"),
        (dict(n_components=0), "n_components must be >= 1"),
        (dict(min_dist=2.0), "min_dist must be <= spread"),
        (dict(set_op_mix_ratio=1.5), "set_op_mix_ratio"),
        (dict(negative_sample_rate=0), "negative_sample_rate must be >= 1"),
        (dict(local_connectivity=-1.0), "local_connectivity"),
        (dict(approx_knn_iters=0), "approx_knn_iters"),
    ],
)
def test_parameter_validation_messages(kwargs, msg):
    x = workloads.reference_synthetic(32, 6)
    with pytest.raises(ValueError, match=msg):
        Umap(**kwargs).fit(x)


def test_empty_and_single_sample_inputs():
    with pytest.raises(ValueError, match="input data is empty"):
        Umap().fit(np.zeros((0, 3), np.float32))
    with pytest.raises(ValueError, match="need at least two samples"):
        Umap().fit(np.zeros((1, 3), np.float32))
    # the binding rejects zero columns before the core sees the rows
    # (ensure_nonzero_columns, umap_rs/src/lib.rs:166-178)
    with pytest.raises(ValueError, match="data must have at least one column"):
        Umap().fit(np.zeros((40, 0), np.float32))


def test_dense_input_must_be_two_dimensional():
    with pytest.raises(ValueError, match="2D"):
        Umap().fit(np.zeros(10, np.float32))


def test_precomputed_knn_validation_errors():
    x = workloads.reference_synthetic(40, 6)
    idx = np.tile(np.arange(12), (40, 1)).astype(np.int64)
    dist = np.tile(np.linspace(0, 1, 12, dtype=np.float32), (40, 1))
    m = Umap(n_neighbors=10)
    with pytest.raises(ValueError, match="precomputed knn metric"):
        Umap(n_neighbors=10, metric="cosine").fit_transform_with_knn(x, idx, dist)
    with pytest.raises(ValueError, match="identical shapes"):
        m.fit_transform_with_knn(x, idx[:, :11], dist)
    with pytest.raises(ValueError, match="row count must match"):
        m.fit_transform_with_knn(x, idx[:30], dist[:30])
    with pytest.raises(ValueError, match="columns must be >= n_neighbors"):
        m.fit_transform_with_knn(x, idx[:, :5], dist[:, :5])
    bad = dist.copy()
    bad[0, 2] = np.nan
    with pytest.raises(ValueError, match="finite"):
        m.fit_transform_with_knn(x, idx, bad)
    neg = idx.copy()
    neg[0, 1] = -1
    with pytest.raises(ValueError, match="non-negative"):
        m.fit_transform_with_knn(x, neg, dist)
    unsorted = dist.copy()
    unsorted[0, [2, 5]] = unsorted[0, [5, 2]]
    with pytest.raises(ValueError, match="non-decreasing"):
        m.fit_transform_with_knn(x, idx, unsorted)
    dup = idx.copy()
    dup[3, 4] = dup[3, 3]
    with pytest.raises(ValueError, match="duplicate index"):
        m.fit_transform_with_knn(x, dup, dist)
    oob = idx.copy()
    oob[2, 1] = 400
    with pytest.raises(ValueError, match="out of range"):
        m.fit_transform_with_knn(x, oob, dist)


def test_out_buffer_contract():
    x = workloads.reference_synthetic(40, 6)
    m = Umap(n_neighbors=8)
    with pytest.raises(TypeError, match="float32"):
        m.fit_transform(x, out=np.zeros((40, 2), np.float64))
    with pytest.raises(ValueError, match="shape mismatch"):
        m.fit_transform(x, out=np.zeros((39, 2), np.float32))
    with pytest.raises(ValueError, match="C-contiguous"):
        m.fit_transform(x, out=np.zeros((2, 40), np.float32).T)
    with pytest.raises(TypeError, match="ndarray"):
        m.fit_transform(x, out=[[0.0, 0.0]] * 40)


def test_transform_requires_fit():
    with pytest.raises(RuntimeError, match="not fitted"):
        Umap().transform(np.zeros((3, 4), np.float32))


def test_sparse_input_checks_run_before_the_device():
    """The facade's sparse routing (umapers/_api.py:562-632) and the checks of
    sparse_csr_from_py / SparseCsrMatrix::new / the sparse fit
    (umap_rs/src/lib.rs:242-351, rust_umap/src/sparse.rs:20-105,
    rust_umap/src/lib.rs:2241-2258) raise before any device work."""
    sp = pytest.importorskip("scipy.sparse")
    x = sp.random(50, 20, density=0.1, format="csr", dtype=np.float32, random_state=3)
    with pytest.raises(ValueError, match="densmap and output_dens currently support dense"):
        Umap(densmap=True).fit(x)
    with pytest.raises(ValueError, match="categorical supervised UMAP currently supports dense"):
        Umap(target_metric="categorical").fit(x, y=np.zeros(50))
    core = UmapCore(n_neighbors=5)
    ip = np.array([0, 2, 3], np.int64)
    with pytest.raises(ValueError, match="indices must contain non-negative integers"):
        core.fit_sparse_csr(ip, np.array([0, -1, 2]), np.ones(3, np.float32), 4)
    with pytest.raises(ValueError, match="indptr cannot be empty"):
        core.fit_sparse_csr(np.array([], np.int64), np.array([], np.int64),
                            np.array([], np.float32), 4)
    with pytest.raises(ValueError, match=r"csr indptr last value \(3\) must equal nnz \(2\)"):
        core.fit_sparse_csr(ip, np.array([0, 1]), np.ones(2, np.float32), 4)
    with pytest.raises(ValueError, match="csr indices/data lengths must match"):
        core.fit_sparse_csr(ip, np.array([0, 1, 2]), np.ones(2, np.float32), 4)
    with pytest.raises(ValueError, match="csr row 0 indices must be strictly increasing"):
        core.fit_sparse_csr(ip, np.array([1, 1, 2]), np.ones(3, np.float32), 4)
    with pytest.raises(ValueError, match="csr row 1 has column index 4 out of bounds for n_cols=4"):
        core.fit_sparse_csr(ip, np.array([0, 1, 4]), np.ones(3, np.float32), 4)
    with pytest.raises(ValueError, match="csr data must be finite"):
        core.fit_sparse_csr(ip, np.array([0, 1, 2]), np.array([1, np.nan, 1], np.float32), 4)
    with pytest.raises(ValueError, match="csr indptr must be non-decreasing"):
        core.fit_sparse_csr(np.array([0, 3, 2, 3]), np.array([0, 1, 2]), np.ones(3, np.float32), 4)
    with pytest.raises(ValueError, match="input data is empty"):
        core.fit_sparse_csr(np.array([0], np.int64), np.array([], np.int64),
                            np.array([], np.float32), 4)
    with pytest.raises(ValueError, match="Canberra metric is currently supported for dense input"):
        Umap(metric="canberra", n_neighbors=5).fit(x)
    with pytest.raises(ValueError, match="n_neighbors above 32"):
        Umap(n_neighbors=40).fit(x)


def test_supervised_target_checks_run_before_the_device():
    # validate_supervised_target (rust_umap/src/lib.rs:2260-2283) and the
    # facade's label conversion (_api.py:127-131), before any device work
    x = np.zeros((50, 3), np.float32)
    with pytest.raises(ValueError, match=r"target label length \(49\) must match number of "
                                         r"samples \(50\)"):
        Umap(target_metric="categorical").fit(x, y=np.zeros(49))
    with pytest.raises(ValueError, match="y must be a 1D label array, got ndim=2"):
        Umap(target_metric="categorical").fit_transform(x, y=np.zeros((50, 1)))
    core = UmapCore(n_neighbors=5)
    with pytest.raises(ValueError, match=r"target_weight must be finite and in \[0, 1\]"):
        core.fit_supervised(x, np.zeros(50), 1.5)
    with pytest.raises(ValueError, match=r"target_weight must be finite and in \[0, 1\]"):
        core.fit_transform_supervised(x, np.zeros(50), float("nan"))
    with pytest.raises(ValueError, match="target_n_neighbors must be >= 1 when provided"):
        core.fit_supervised(x, np.zeros(50), 0.5, 0)
    with pytest.raises(OverflowError):
        core.fit_supervised(x, np.zeros(50), 0.5, -3)
    with pytest.raises(ValueError, match="target_weight must be finite and in"):
        Umap(target_metric="categorical", target_weight=2.0)


def test_inverse_transform_needs_a_fit():
    # inverse_transform_requires_fit (rust_umap/src/lib.rs:6366-6374) and the
    # facade's out= check (_api.py:866-871), before any device work
    with pytest.raises(RuntimeError, match="model is not fitted yet"):
        Umap().inverse_transform(np.array([[0.1, 0.2]], np.float32))
    with pytest.raises(RuntimeError, match="model must be fit before inverse_transform"):
        Umap().inverse_transform(np.zeros((1, 2), np.float32), out=np.zeros((1, 3), np.float32))
    with pytest.raises(RuntimeError, match="model is not fitted yet"):
        UmapCore().inverse_transform(np.zeros((1, 2), np.float32))


def test_metrics_outside_the_engine_are_rejected_at_fit():
    x = workloads.reference_synthetic(40, 6)
    with pytest.raises(ValueError, match="not supported by the B200 engine"):
        Umap(metric="manhattan", n_neighbors=8).fit(x)


def test_umapcore_is_importable_from_the_drop_in_path():
    core = UmapCore(n_neighbors=12, n_components=3)
    assert core.n_neighbors == 12 and core.n_components == 3 and core.n_features is None
    assert core.embedding is None
    assert umapers.__version__.startswith("1.")
