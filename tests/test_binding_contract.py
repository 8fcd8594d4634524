"""The Python binding contract of the reference (umap_rs/tests/test_binding.py),
checked against this package through the drop-in names ``umapers``,
``umapers._api`` and ``umapers._umapers``.

Each test below restates one reference test (cited by line) with its inputs
and assertions.  Tests that fit run on the GPU (marked ``gpu``); pure
construction and validation checks run anywhere.  Reference tests not
restated here, and why:
- the six dense metrics beyond euclidean / cosine (chebyshev, minkowski,
  correlation, canberra, braycurtis, manhattan) are out of this engine's
  scope, so test_expanded_dense_metrics_fit_transform_and_transform (:667),
  test_sparse_csr_expanded_metric_support_and_dense_only_rejection (:1314) and
  test_precomputed_knn_out_buffer_and_metric_variant_work (:1240) are left
  out; the two sparse tests that fit with manhattan only to reach an
  inverse_transform error (:1493, :1516) are restated with euclidean;
- ParametricUmap (:861-918) and AlignedUmap (:921-985) are other estimators;
- plot helpers (:114) and typing stubs (:87) are packaging outside the path;
- the umap-learn comparison (:740) needs umap-learn, which is not installed.
"""
import importlib
import inspect
import subprocess
import sys

import numpy as np
import pytest

import umapers._api as api
from umapers import Umap, fit_transform
from umapers._umapers import UmapCore
from umapers_b200 import workloads

gpu = pytest.mark.gpu


def make_dataset(n_samples=180, n_features=12, seed=42):
    """The reference tests' three-centre standardised dataset (:27-41)."""
    return workloads.three_centres(n_samples, n_features, seed)


def _small(**kw):
    base = dict(n_components=2, init="random", use_approximate_knn=False)
    base.update(kw)
    return base


# ------------------------------------------------------ surface, no device --
def test_public_api_has_helpful_docstrings():  # :50
    docs = {name: inspect.getdoc(obj) or "" for name, obj in {
        "Umap": Umap, "Umap.__init__": Umap.__init__, "Umap.fit": Umap.fit,
        "Umap.fit_transform": Umap.fit_transform,
        "Umap.fit_transform_with_knn": Umap.fit_transform_with_knn,
        "Umap.transform": Umap.transform, "Umap.inverse_transform": Umap.inverse_transform,
        "fit_transform": fit_transform}.items()}
    for name, doc in docs.items():
        assert doc.strip(), name
    ft = docs["Umap.fit_transform"].lower()
    assert "shape" in ft and "dtype" in ft and "out" in ft
    fk = docs["Umap.fit_transform_with_knn"].lower()
    assert "advanced" in fk and "knn" in fk and "precomputed" in fk
    assert "out" in docs["Umap.transform"].lower()
    assert "out" in docs["Umap.inverse_transform"].lower()


def test_top_level_fit_transform_signature_is_inspectable():  # :79
    sig = inspect.signature(fit_transform)
    assert "data" in sig.parameters and "kwargs" in sig.parameters
    assert sig.parameters["kwargs"].kind is inspect.Parameter.VAR_KEYWORD


def test_import_umapers_does_not_import_optional_ecosystem_dependencies():  # :98
    code = ("import sys; sys.path.insert(0, %r); import umapers; "
            "print('matplotlib' in sys.modules); print('sklearn' in sys.modules)"
            % str(__import__("pathlib").Path(__file__).resolve().parents[1]))
    out = subprocess.run([sys.executable, "-I", "-c", code], check=True, capture_output=True,
                         text=True).stdout
    assert out.splitlines() == ["False", "False"]


def test_default_ann_params_use_quality_tuned_recall_budget():  # :183
    m = Umap()
    assert m.use_approximate_knn is True
    assert (m.approx_knn_candidates, m.approx_knn_iters) == (50, 14)
    p = m.get_params()
    assert (p["approx_knn_candidates"], p["approx_knn_iters"]) == (50, 14)


def test_ann_mode_overrides_legacy_knn_flags(monkeypatch):  # :214
    seen = []

    class RecordingCore:
        def __init__(self, **kwargs):
            seen.append(kwargs)
            self.n_features = None

    monkeypatch.setattr(api, "UmapCore", RecordingCore)
    modes = [api.Umap(ann_mode=mode, use_approximate_knn=legacy, approx_knn_threshold=321)
             for mode, legacy in (("auto", False), ("exact", True), ("approximate", False))]
    assert [m.ann_mode for m in modes] == ["auto", "exact", "approximate"]
    assert (seen[0]["use_approximate_knn"], seen[0]["approx_knn_threshold"]) == (False, 321)
    assert (seen[1]["use_approximate_knn"], seen[1]["approx_knn_threshold"]) == (False, 321)
    assert (seen[2]["use_approximate_knn"], seen[2]["approx_knn_threshold"]) == (True, 0)


def test_ann_mode_rejects_unknown_value():  # :251
    with pytest.raises(ValueError, match="unsupported ann_mode 'hybrid'"):
        Umap(ann_mode="hybrid")


def test_get_params_returns_constructor_arguments():  # :291
    m = Umap(n_neighbors=9, n_components=3, n_epochs=25, metric="cosine", init="random",
             ann_mode="exact", target_metric="categorical", target_weight=0.25,
             target_n_neighbors=5)
    p = m.get_params()
    assert set(p) == set(api._PARAM_NAMES)
    assert (p["n_neighbors"], p["n_components"], p["n_epochs"]) == (9, 3, 25)
    assert (p["metric"], p["ann_mode"], p["use_approximate_knn"]) == ("cosine", "exact", False)
    assert (p["target_metric"], p["target_weight"], p["target_n_neighbors"]) == \
        ("categorical", 0.25, 5)


def test_set_params_rejects_unknown_parameter():  # :346
    with pytest.raises(ValueError, match="Invalid parameter 'unknown'"):
        Umap().set_params(unknown=1)


def test_categorical_supervised_rejects_invalid_target_parameters():  # :510
    with pytest.raises(ValueError, match="unsupported target_metric 'continuous'"):
        Umap(target_metric="continuous")
    with pytest.raises(ValueError, match=r"target_weight must be finite and in \[0, 1\]"):
        Umap(target_metric="categorical", target_weight=1.1)
    with pytest.raises(ValueError, match="target_n_neighbors must be >= 1"):
        Umap(target_metric="categorical", target_n_neighbors=0)


def test_unsupported_metric_and_init_are_rejected():  # :659
    with pytest.raises(ValueError, match="unsupported metric 'hamming'"):
        Umap(metric="hamming")
    with pytest.raises(ValueError, match="unsupported init 'pca'"):
        Umap(init="pca")


def test_expanded_metric_kwds_validation():  # :699
    with pytest.raises(ValueError, match="requires metric_kwds"):
        Umap(metric="minkowski")
    with pytest.raises(ValueError, match="finite and > 0"):
        Umap(metric="minkowski", metric_kwds={"p": 0.0})
    with pytest.raises(ValueError, match="unsupported metric_kwds for minkowski: w"):
        Umap(metric="minkowski", metric_kwds={"p": 2.0, "w": [1.0, 2.0]})
    with pytest.raises(ValueError, match="unsupported metric_kwds for euclidean: p"):
        Umap(metric="euclidean", metric_kwds={"p": 2.0})


def test_densmap_rejects_invalid_params():  # :837 (parameter part)
    with pytest.raises(ValueError, match="dens_lambda must be finite and >= 0"):
        Umap(dens_lambda=-1.0)
    with pytest.raises(ValueError, match=r"dens_frac must be finite and in \[0, 1\]"):
        Umap(dens_frac=1.5)
    with pytest.raises(ValueError, match="dens_var_shift must be finite and > 0"):
        Umap(dens_var_shift=0.0)


def test_transform_and_inverse_transform_require_fit():  # :1073
    m = Umap(**_small(n_neighbors=10, n_epochs=20, random_seed=33))
    with pytest.raises(RuntimeError, match="model is not fitted yet"):
        m.transform(np.zeros((8, 6), np.float32))
    with pytest.raises(RuntimeError, match="model is not fitted yet"):
        m.inverse_transform(np.zeros((8, 2), np.float32))
    with pytest.raises(RuntimeError, match=r"model must be fit before inverse_transform\(out=\.\.\.\)"):
        m.inverse_transform(np.zeros((8, 2), np.float32), out=np.empty((8, 6), np.float32))


def test_binding_getters_before_fit():  # :1538 (before the fit)
    m = Umap(**_small(n_neighbors=9, n_epochs=30, random_seed=67))
    assert (m.n_neighbors, m.n_components) == (9, 2)
    assert m._core.n_features is None


# ----------------------------------------------------------- fits (GPU) --
@gpu
def test_trustworthiness_report_uses_optional_sklearn():  # :127
    diagnostics = importlib.import_module("umapers.diagnostics")
    x = make_dataset(48, 6, 62)
    emb = Umap(**_small(n_neighbors=6, n_epochs=20, random_seed=47)).fit_transform(x)
    r = diagnostics.trustworthiness_report(x, emb, n_neighbors=5)
    assert (r["n_samples"], r["n_features"], r["n_components"], r["n_neighbors"]) == \
        (x.shape[0], x.shape[1], 2, 5)
    assert 0.0 <= r["trustworthiness"] <= 1.0


@gpu
def test_fit_transform_out_buffer_and_inverse_roundtrip():  # :153
    x = make_dataset()
    m = Umap(**_small(n_neighbors=12, n_epochs=80, metric="euclidean", random_seed=7))
    out = np.empty((x.shape[0], 2), np.float32)
    emb = m.fit_transform(x, out=out)
    assert emb is out and emb.dtype == np.float32 and np.all(np.isfinite(emb))
    t = m.transform(x[:24])
    r = m.inverse_transform(t)
    assert t.shape == (24, 2) and r.shape == (24, x.shape[1])
    assert np.all(np.isfinite(t)) and np.all(np.isfinite(r))


@gpu
def test_profile_fit_transform_reports_stage_timings():  # :194
    x = make_dataset(72, 6, 83)
    prof = Umap(n_neighbors=8, n_components=2, n_epochs=20, random_seed=31,
                init="random").profile_fit_transform(x)
    assert prof["embedding"].shape == (72, 2) and np.all(np.isfinite(prof["embedding"]))
    assert (prof["n_samples"], prof["n_features"], prof["n_epochs"]) == (72, 6, 20)
    assert prof["n_edges"] > 0 and prof["used_approximate_knn"] is False
    t = prof["timings"]
    assert t["total_sec"] > 0.0 and t["knn_sec"] >= 0.0 and t["optimize_sec"] >= 0.0


@gpu
def test_knn_diagnostics_reports_ann_recall_and_sets_attribute():  # :256
    x = make_dataset(96, 8, 61)
    m = Umap(**_small(n_neighbors=8, n_epochs=20, metric="euclidean", random_seed=45,
                      ann_mode="approximate", approx_knn_candidates=24, approx_knn_iters=7))
    assert not hasattr(m, "knn_diagnostics_")
    d = m.knn_diagnostics(x)
    assert d is m.knn_diagnostics_
    assert (d["n_samples"], d["n_features"], d["n_neighbors"], d["metric"]) == \
        (96, 8, 8, "euclidean")
    assert d["candidate_pool"] >= 8 and d["n_iters"] == 7
    assert d["mean_recall"] >= d["worst_decile_recall"]
    assert d["worst_decile_recall"] + 1e-6 >= d["min_recall"]
    assert d["mean_recall"] >= 0.60
    pr = d["per_row_recall"]
    assert pr.shape == (96,) and pr.dtype == np.float32 and np.all((pr >= 0) & (pr <= 1))
    m.set_params(n_neighbors=9)
    assert not hasattr(m, "knn_diagnostics_")


@gpu
def test_set_params_rebuilds_core_and_clears_fitted_attributes():  # :318
    x = make_dataset(48, 6, 80)
    m = Umap(**_small(n_neighbors=6, n_epochs=20, random_seed=69))
    m.fit(x)
    core = m._core
    assert (m.n_features_in_, m.n_samples_fit_, m.embedding_.shape) == (6, 48, (48, 2))
    assert m.set_params(n_neighbors=7, target_metric="categorical", target_weight=0.2) is m
    assert (m.n_neighbors, m.target_metric, m.target_weight) == (7, "categorical", 0.2)
    assert m._core is not core
    for attr in ("embedding_", "n_features_in_", "n_samples_fit_"):
        assert not hasattr(m, attr)


@gpu
def test_sklearn_clone_and_pipeline_smoke():  # :351 (euclidean: minkowski is out of scope)
    from sklearn.base import clone
    from sklearn.pipeline import Pipeline
    from sklearn.preprocessing import FunctionTransformer

    x = make_dataset(60, 7, 81)
    m = Umap(**_small(n_neighbors=6, n_epochs=20, random_seed=77))
    c = clone(m)
    assert isinstance(c, Umap) and c.get_params() == m.get_params()
    assert not hasattr(c, "embedding_")
    pipe = Pipeline([("umap", m), ("identity", FunctionTransformer(validate=False))])
    emb = pipe.fit_transform(x)
    assert emb.shape == (60, 2) and np.all(np.isfinite(emb))
    assert pipe.get_params()["umap__n_neighbors"] == 6
    # a clone of an estimator configured with an out-of-scope metric keeps its parameters
    mk = Umap(metric="minkowski", metric_kwds={"p": 3.0})
    assert clone(mk).get_params() == mk.get_params()


@gpu
def test_target_metric_none_with_y_is_noop():  # :390
    x = make_dataset(72, 8, 82)
    y = np.arange(72, dtype=np.int64) % 3
    params = _small(n_neighbors=8, n_epochs=30, random_seed=71)
    base = Umap(**params).fit_transform(x)
    with_y = Umap(**params, target_metric=None).fit_transform(x, y)
    np.testing.assert_array_equal(with_y, base)


@gpu
def test_categorical_target_weight_zero_matches_unsupervised():  # :408
    x = make_dataset(72, 8, 83)
    y = np.arange(72, dtype=np.int64) % 3
    params = _small(n_neighbors=8, n_epochs=30, random_seed=73)
    base = Umap(**params).fit_transform(x)
    zero = Umap(**params, target_metric="categorical", target_weight=0.0).fit_transform(x, y)
    np.testing.assert_array_equal(zero, base)


@gpu
def test_categorical_supervised_fit_transform_changes_embedding_and_supports_out():  # :426
    x = make_dataset(84, 8, 84)
    y = np.where(np.arange(84) < 42, 0, 1).astype(np.int64)
    y[::7] = -1
    params = _small(n_neighbors=8, n_epochs=30, random_seed=79)
    base = Umap(**params).fit_transform(x)
    out = np.empty((84, 2), np.float32)
    sup = Umap(**params, target_metric="categorical", target_weight=0.7,
               target_n_neighbors=4).fit_transform(x, y, out=out)
    assert sup is out and sup.shape == base.shape and sup.dtype == np.float32
    assert np.all(np.isfinite(sup)) and not np.array_equal(sup, base)


@gpu
def test_categorical_supervised_fit_supports_dense_input():  # :455
    x = make_dataset(48, 6, 85)
    y = np.arange(48, dtype=np.int64) % 2
    m = Umap(**_small(n_neighbors=6, n_epochs=20, random_seed=81, target_metric="categorical"))
    assert m.fit(x, y) is m
    assert m._core.n_features == 6


@gpu
def test_categorical_supervised_rejects_sparse_input():  # :473
    import scipy.sparse as sp

    x = make_dataset(48, 6, 86)
    x[x < 0.1] = 0.0
    y = np.arange(48, dtype=np.int64) % 2
    m = Umap(**_small(n_neighbors=6, n_epochs=20, random_seed=83, target_metric="categorical"))
    with pytest.raises(ValueError,
                       match="categorical supervised UMAP currently supports dense input only"):
        m.fit_transform(sp.csr_matrix(x), y)


@gpu
def test_categorical_supervised_rejects_label_length_mismatch():  # :493
    x = make_dataset(48, 6, 87)
    m = Umap(**_small(n_neighbors=6, n_epochs=20, random_seed=85, target_metric="categorical"))
    with pytest.raises(ValueError, match="target label length"):
        m.fit_transform(x, np.zeros(47, np.int64))


@gpu
def test_transform_and_inverse_transform_support_out_buffers():  # :521
    x = make_dataset(120, 10, 21)
    m = Umap(**_small(n_neighbors=10, n_epochs=60, metric="euclidean", random_seed=17))
    m.fit(x)
    t_out = np.empty((18, 2), np.float32)
    t = m.transform(x[:18], out=t_out)
    assert t is t_out and np.all(np.isfinite(t))
    r_out = np.empty((18, 10), np.float32)
    r = m.inverse_transform(t, out=r_out)
    assert r is r_out and r.shape == (18, 10) and np.all(np.isfinite(r))


@gpu
def test_inverse_transform_empty_input_preserves_feature_width():  # :547
    x = make_dataset(96, 11, 25)
    m = Umap(**_small(n_neighbors=10, n_epochs=50, metric="euclidean", random_seed=31))
    m.fit(x)
    empty = np.empty((0, 2), np.float32)
    assert m.inverse_transform(empty).shape == (0, 11)
    out = np.empty((0, 11), np.float32)
    assert m.inverse_transform(empty, out=out) is out


@gpu
def test_precomputed_knn_path_consistency():  # :570
    from sklearn.manifold import trustworthiness
    from sklearn.neighbors import NearestNeighbors

    x = make_dataset(160, 10, 123)
    k = 10
    dist, idx = NearestNeighbors(n_neighbors=k + 1, algorithm="brute").fit(x).kneighbors(x)
    ki, kd = idx[:, 1:].astype(np.int64), dist[:, 1:].astype(np.float32)
    params = _small(n_neighbors=k, n_epochs=60, metric="euclidean", random_seed=11)
    e1 = Umap(**params).fit_transform(x)
    e2 = Umap(**params).fit_transform_with_knn(x, ki, kd, knn_metric="euclidean")
    assert e1.shape == e2.shape and np.all(np.isfinite(e1)) and np.all(np.isfinite(e2))
    t1 = trustworthiness(x, e1, n_neighbors=k)
    t2 = trustworthiness(x, e2, n_neighbors=k)
    assert abs(t1 - t2) < 0.05


@gpu
def test_umap_core_precomputed_accepts_noncontiguous_knn_buffers():  # :608
    x = make_dataset(64, 6, 35)
    k = 8
    ib = np.full((64, 2 * k), -1, np.int64)
    ib[:, ::2] = np.tile(np.arange(k, dtype=np.int64), (64, 1))
    db = np.empty((64, 2 * k), np.float32)
    db[:, ::2] = np.tile(np.arange(k, dtype=np.float32), (64, 1))
    ki, kd = ib[:, ::2], db[:, ::2]
    assert not ki.flags.c_contiguous and not kd.flags.c_contiguous
    core = UmapCore(n_neighbors=k, n_components=2, n_epochs=20, metric="euclidean",
                    init="random", random_seed=39, use_approximate_knn=False)
    emb = core.fit_transform_with_knn(x, ki, kd, knn_metric="euclidean")
    assert emb.shape == (64, 2) and emb.dtype == np.float32 and np.all(np.isfinite(emb))


def _precomputed_model(k, seed):
    return Umap(**_small(n_neighbors=k, n_epochs=20, random_seed=seed))


@gpu
def test_precomputed_knn_rejects_non_finite_distances_early():  # :639
    x = make_dataset(48, 6, 31)
    ki = np.tile(np.arange(8, dtype=np.int64), (48, 1))
    kd = np.ones((48, 8), np.float32)
    kd[0, 0] = np.nan
    with pytest.raises(ValueError, match="knn_dists must contain only finite values"):
        _precomputed_model(8, 5).fit_transform_with_knn(x, ki, kd, knn_metric="euclidean")


@gpu
def test_output_dens_returns_embedding_and_radii():  # :713
    x = make_dataset(64, 8, 90)
    m = Umap(**_small(n_neighbors=8, n_epochs=30, random_seed=95, output_dens=True))
    emb, ro, re = m.fit_transform(x)
    assert emb.shape == (64, 2) and ro.shape == (64,) and re.shape == (64,)
    assert m.embedding_ is emb
    for a, b in ((m.rad_orig_, ro), (m.rad_emb_, re), (m.radii_original_, ro),
                 (m.radii_embedding_, re)):
        assert np.array_equal(a, b)
    assert np.all(np.isfinite(ro)) and np.all(np.isfinite(re))


@gpu
def test_density_attributes_follow_output_dens_lifecycle():  # :784
    x = make_dataset(64, 8, 96)
    attrs = ("rad_orig_", "rad_emb_", "radii_original_", "radii_embedding_")
    m = Umap(n_neighbors=8, n_components=2, n_epochs=30, init="random", random_seed=99,
             densmap=True, output_dens=False)
    assert m.fit_transform(x).shape == (64, 2)
    assert not any(hasattr(m, a) for a in attrs)
    m.set_params(output_dens=True)
    assert not any(hasattr(m, a) for a in attrs)
    emb, ro, re = m.fit_transform(x)
    assert m.rad_orig_ is ro and m.rad_emb_ is re
    assert m.radii_original_ is ro and m.radii_embedding_ is re
    assert emb.shape == (64, 2)
    m.set_params(output_dens=False, densmap=False)
    assert not any(hasattr(m, a) for a in attrs)
    assert m.fit_transform(x).shape == (64, 2)
    assert not any(hasattr(m, a) for a in attrs)


@gpu
def test_densmap_lambda_zero_matches_standard_umap():  # :820
    x = make_dataset(64, 8, 92)
    params = _small(n_neighbors=8, n_epochs=30, random_seed=97)
    standard = Umap(**params).fit_transform(x)
    zero = Umap(**params, densmap=True, dens_lambda=0.0).fit_transform(x)
    np.testing.assert_array_equal(zero, standard)


@gpu
def test_densmap_rejects_out_buffer_with_output_dens():  # :837 (out= part)
    x = make_dataset(32, 6, 94)
    m = Umap(**_small(n_neighbors=6, n_epochs=20, random_seed=99, output_dens=True))
    with pytest.raises(ValueError, match="out cannot be used when output_dens=True"):
        m.fit_transform(x, out=np.empty((32, 2), np.float32))


@gpu
def test_precomputed_knn_rejects_shape_mismatch_early():  # :988
    x = make_dataset(48, 6, 37)
    ki = np.tile(np.arange(8, dtype=np.int64), (48, 1))
    kd = np.ones((48, 7), np.float32)
    with pytest.raises(ValueError, match="knn_indices and knn_dists must have identical shapes"):
        _precomputed_model(8, 7).fit_transform_with_knn(x, ki, kd, knn_metric="euclidean")


@gpu
def test_precomputed_knn_rejects_negative_indices_early():  # :1007
    x = make_dataset(48, 6, 41)
    ki = np.tile(np.arange(8, dtype=np.int64), (48, 1))
    ki[0, 0] = -1
    kd = np.ones((48, 8), np.float32)
    with pytest.raises(ValueError, match="knn indices must be non-negative integers"):
        _precomputed_model(8, 9).fit_transform_with_knn(x, ki, kd, knn_metric="euclidean")


@gpu
def test_non_float32_and_non_contiguous_input_is_normalized():  # :1027
    x = np.asfortranarray(make_dataset(100, 8, 5).astype(np.float64))
    emb = Umap(**_small(n_neighbors=10, n_epochs=40, metric="euclidean",
                        random_seed=13)).fit_transform(x)
    assert emb.dtype == np.float32 and emb.flags.c_contiguous and emb.shape == (100, 2)


@gpu
def test_fit_transform_rejects_invalid_out_buffers():  # :1047
    x = make_dataset(96, 8, 15)
    m = Umap(**_small(n_neighbors=10, n_epochs=40, metric="euclidean", random_seed=27))
    with pytest.raises(TypeError, match="out dtype must be float32"):
        m.fit_transform(x, out=np.empty((96, 2), np.float64))
    with pytest.raises(ValueError, match="out must be C-contiguous"):
        m.fit_transform(x, out=np.empty((96, 2), np.float32, order="F"))
    ro = np.empty((96, 2), np.float32)
    ro.setflags(write=False)
    with pytest.raises(ValueError, match="out must be writeable"):
        m.fit_transform(x, out=ro)


@gpu
def test_transform_and_inverse_transform_reject_invalid_out_buffers():  # :1096
    x = make_dataset(96, 8, 18)
    m = Umap(**_small(n_neighbors=10, n_epochs=40, metric="euclidean", random_seed=37))
    m.fit(x)
    q = x[:12]
    emb = m.transform(q)
    for call, shape in ((lambda o: m.transform(q, out=o), (12, 2)),
                        (lambda o: m.inverse_transform(emb, out=o), (12, 8))):
        with pytest.raises(TypeError, match="out dtype must be float32"):
            call(np.empty(shape, np.float64))
        with pytest.raises(ValueError, match="out must be C-contiguous"):
            call(np.empty(shape, np.float32, order="F"))
        ro = np.empty(shape, np.float32)
        ro.setflags(write=False)
        with pytest.raises(ValueError, match="out must be writeable"):
            call(ro)


@gpu
def test_zero_column_data_is_rejected_with_value_error():  # :1139
    x = np.empty((16, 0), np.float32)
    m = Umap(**_small(n_neighbors=5, n_epochs=20, random_seed=3))
    with pytest.raises(ValueError, match="data must have at least one column"):
        m.fit(x)
    with pytest.raises(ValueError, match="data must have at least one column"):
        m.fit_transform(x)


@gpu
def test_zero_column_precomputed_knn_is_rejected_with_value_error():  # :1157
    x = make_dataset(40, 6, 9)
    m = Umap(**_small(n_neighbors=6, n_epochs=20, random_seed=19))
    with pytest.raises(ValueError, match="knn columns must be >= n_neighbors"):
        m.fit_transform_with_knn(x, np.empty((40, 0), np.int64), np.empty((40, 0), np.float32),
                                 knn_metric="euclidean")


@gpu
def test_precomputed_knn_rejects_row_count_mismatch_early():  # :1175
    x = make_dataset(40, 6, 43)
    ki = np.tile(np.arange(8, dtype=np.int64), (39, 1))
    kd = np.ones((39, 8), np.float32)
    with pytest.raises(ValueError, match="knn row count must match data row count"):
        _precomputed_model(8, 41).fit_transform_with_knn(x, ki, kd, knn_metric="euclidean")


@gpu
def test_precomputed_knn_rejects_negative_distances_early():  # :1194
    x = make_dataset(48, 6, 45)
    ki = np.tile(np.arange(8, dtype=np.int64), (48, 1))
    kd = np.ones((48, 8), np.float32)
    kd[0, 0] = -0.1
    with pytest.raises(ValueError, match="knn_dists must be non-negative"):
        _precomputed_model(8, 43).fit_transform_with_knn(x, ki, kd, knn_metric="euclidean")


@gpu
def test_precomputed_knn_disable_validation_still_rejects_invalid_distances_in_core():  # :1214
    x = make_dataset(48, 6, 47)
    ki = np.tile(np.arange(8, dtype=np.int64), (48, 1))
    kd = np.ones((48, 8), np.float32)
    kd[0, 0] = -0.1
    with pytest.raises(ValueError, match="precomputed knn distance must be finite and >= 0"):
        _precomputed_model(8, 47).fit_transform_with_knn(x, ki, kd, knn_metric="euclidean",
                                                         validate_precomputed=False)


@gpu
def test_precomputed_knn_non_contiguous_arrays_fallback_to_dense_row_path():  # :1269
    from sklearn.neighbors import NearestNeighbors

    x = make_dataset(96, 8, 50)
    dist, idx = NearestNeighbors(n_neighbors=11, algorithm="brute").fit(x).kneighbors(x)
    ki = np.asfortranarray(idx[:, 1:].astype(np.int64))
    kd = np.asfortranarray(dist[:, 1:].astype(np.float32))
    emb = Umap(**_small(n_neighbors=10, n_epochs=40, random_seed=57)).fit_transform_with_knn(
        x, ki, kd, knn_metric="euclidean")
    assert emb.shape == (96, 2) and np.all(np.isfinite(emb))


@gpu
def test_precomputed_knn_rejects_invalid_metric():  # :1295
    x = make_dataset(40, 6, 51)
    ki = np.tile(np.arange(8, dtype=np.int64), (40, 1))
    kd = np.ones((40, 8), np.float32)
    with pytest.raises(ValueError, match="unsupported metric 'hamming'"):
        _precomputed_model(8, 59).fit_transform_with_knn(x, ki, kd, knn_metric="hamming")


def _sparse(n, d, seed, cut):
    import scipy.sparse as sp

    x = make_dataset(n, d, seed)
    x[x < cut] = 0.0
    return x, sp.csr_matrix(x)


@gpu
def test_sparse_csr_rejects_densmap_and_output_dens():  # :1356
    _, xs = _sparse(40, 8, 57, 0.15)
    with pytest.raises(ValueError, match="dense input only"):
        Umap(**_small(n_neighbors=6, n_epochs=20, random_seed=101, densmap=True)).fit_transform(xs)
    with pytest.raises(ValueError, match="dense input only"):
        Umap(**_small(n_neighbors=6, n_epochs=20, random_seed=103, output_dens=True)).fit(xs)


@gpu
def test_sparse_csr_fit_transform_and_dense_transform_out_buffer():  # :1386
    x, xs = _sparse(90, 14, 55, 0.15)
    m = Umap(**_small(n_neighbors=8, n_epochs=50, metric="cosine", random_seed=23))
    out = np.empty((90, 2), np.float32)
    emb = m.fit_transform(xs, out=out)
    assert emb is out and np.all(np.isfinite(emb))
    t_out = np.empty((12, 2), np.float32)
    t = m.transform(x[:12], out=t_out)
    assert t is t_out and np.all(np.isfinite(t))


@gpu
def test_sparse_csr_fit_supports_sparse_query_transform():  # :1416
    import scipy.sparse as sp

    x, xs = _sparse(84, 16, 58, 0.2)
    m = Umap(**_small(n_neighbors=7, n_epochs=40, metric="cosine", random_seed=37))
    m.fit_transform(xs)
    dense_t = m.transform(x[:11])
    sparse_t = m.transform(sp.csr_matrix(x[:11]))
    assert sparse_t.shape == dense_t.shape
    np.testing.assert_allclose(sparse_t, dense_t, rtol=1e-6, atol=1e-6)
    out = np.empty((11, 2), np.float32)
    got = m.transform(sp.csr_matrix(x[:11]), out=out)
    assert got is out
    np.testing.assert_allclose(got, dense_t, rtol=1e-6, atol=1e-6)


@gpu
def test_sparse_csc_and_coo_inputs_normalize_to_csr():  # :1448
    import scipy.sparse as sp

    x = make_dataset(72, 12, 59)
    x[x < 0.2] = 0.0
    m = Umap(**_small(n_neighbors=7, n_epochs=35, metric="euclidean", random_seed=41))
    emb = m.fit_transform(sp.csc_matrix(x))
    dense_t = m.transform(x[:9])
    coo_t = m.transform(sp.coo_matrix(x[:9]))
    assert emb.shape == (72, 2) and np.all(np.isfinite(emb)) and coo_t.shape == dense_t.shape
    np.testing.assert_allclose(coo_t, dense_t, rtol=1e-6, atol=1e-6)


@gpu
def test_sparse_query_after_dense_fit_is_explicitly_unsupported():  # :1476
    import scipy.sparse as sp

    x = make_dataset(64, 10, 60)
    m = Umap(**_small(n_neighbors=6, n_epochs=30, random_seed=43)).fit(x)
    with pytest.raises(ValueError,
                       match="sparse query transform is supported only for sparse-fitted models"):
        m.transform(sp.csr_matrix(x[:5]))


@gpu
def test_sparse_csr_fit_tracks_feature_count_for_inverse_out_error():  # :1493 (euclidean)
    _, xs = _sparse(64, 9, 71, 0.2)
    m = Umap(**_small(n_neighbors=6, n_epochs=40, metric="euclidean", random_seed=29))
    m.fit(xs)
    with pytest.raises(ValueError, match="output buffer shape mismatch"):
        m.inverse_transform(np.zeros((5, 2), np.float32), out=np.empty((5, 10), np.float32))


@gpu
def test_sparse_trained_inverse_transform_is_explicitly_unsupported():  # :1516 (euclidean)
    _, xs = _sparse(64, 9, 73, 0.2)
    m = Umap(**_small(n_neighbors=6, n_epochs=40, metric="euclidean", random_seed=61))
    m.fit(xs)
    with pytest.raises(ValueError,
                       match="inverse_transform is not supported for sparse-trained models yet"):
        m.inverse_transform(np.zeros((5, 2), np.float32))


@gpu
def test_binding_getters_track_feature_count_after_fit():  # :1538
    x = make_dataset(72, 7, 79)
    m = Umap(**_small(n_neighbors=9, n_epochs=30, random_seed=67))
    assert m._core.n_features is None
    m.fit(x)
    assert m._core.n_features == 7
