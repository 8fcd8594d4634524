"""End-to-end Umap behaviour on the GPU (the reference's fit/transform
contract tests, rust_umap/src/lib.rs:5953-6236, 7696-7732, and
umap_rs/tests/test_binding.py)."""
import numpy as np
import pytest

import umapers
from umapers import Umap
from umapers_b200 import diagnostics, workloads

pytestmark = pytest.mark.gpu


def test_fit_transform_shape_and_finite():
    x = workloads.reference_synthetic(80, 8)
    emb = Umap(n_neighbors=12, n_epochs=60, init="random", random_seed=7).fit_transform(x)
    assert emb.shape == (80, 2) and emb.dtype == np.float32 and np.all(np.isfinite(emb))


def test_fit_sets_attributes_and_out_buffers():
    x = workloads.three_centres()
    m = Umap(n_neighbors=10)
    out = np.empty((180, 2), np.float32)
    assert m.fit_transform(x, out=out) is out
    assert m.n_features_in_ == 12 and m.n_samples_fit_ == 180
    np.testing.assert_array_equal(m.embedding_, out)
    m2 = Umap(n_neighbors=10).fit(x)
    assert m2.embedding_.shape == (180, 2)


def test_profile_fit_transform_reports_stage_timings():
    x = workloads.three_centres(400, 16)
    r = Umap(n_neighbors=12).profile_fit_transform(x)
    for key in ("validation_sec", "knn_sec", "smooth_knn_sec", "symmetrize_sec", "init_sec",
                "optimize_sec", "total_sec"):
        assert key in r["timings"] and r["timings"][key] >= 0.0
    assert r["embedding"].shape == (400, 2) and r["n_edges"] > 0 and r["n_epochs"] == 500
    assert r["used_approximate_knn"] is False


def test_ann_switch_follows_threshold():
    x = workloads.isotropic_mixture(500, 16, 4, 3.0, seed=2)
    exact = Umap(n_neighbors=10, approx_knn_threshold=125, n_epochs=20).profile_fit_transform(x)
    approx = Umap(n_neighbors=10, approx_knn_threshold=124, n_epochs=20).profile_fit_transform(x)
    assert exact["used_approximate_knn"] is False and approx["used_approximate_knn"] is True
    forced = Umap(n_neighbors=10, ann_mode="approximate", n_epochs=20).profile_fit_transform(x)
    assert forced["used_approximate_knn"] is True


def test_precomputed_knn_path_consistency(orc):
    # umap_rs/tests/test_binding.py:570-605: |trust difference| < 0.05
    x = workloads.three_centres(300, 12)
    idx, dist = orc.exact_knn(x, 16)
    m1 = Umap(n_neighbors=15, random_seed=1)
    e1 = m1.fit_transform(x)
    m2 = Umap(n_neighbors=15, random_seed=1)
    e2 = m2.fit_transform_with_knn(x, idx, dist)
    t1 = diagnostics.trustworthiness_report(x, e1)["trustworthiness"]
    t2 = diagnostics.trustworthiness_report(x, e2)["trustworthiness"]
    assert abs(t1 - t2) < 0.05
    # non-self precomputed rows (rust_umap/src/lib.rs:7023-7085)
    e3 = Umap(n_neighbors=15).fit_transform_with_knn(x, idx[:, 1:], dist[:, 1:])
    assert np.all(np.isfinite(e3))


def test_disconnected_components_stay_separated():
    # rust_umap/src/lib.rs:7663-7696, with the reference's bounds.  The layout
    # SGD updates concurrently (Hogwild), so on this 240-point graph a single
    # fit varies more than the reference's sequential one: ten fits on a B200
    # gave separation ratios 1.88-2.58, and one earlier run 1.06.  The bounds
    # hold for the median of three fits.
    x, labels = workloads.disconnected_components(4, 60)
    stats = []
    for _ in range(3):
        emb = Umap(n_neighbors=10, n_epochs=60, random_seed=42, ann_mode="exact").fit_transform(x)
        cents = np.stack([emb[labels == c].mean(0) for c in range(4)])
        min_d = min(np.linalg.norm(cents[i] - cents[j]) for i in range(4) for j in range(i + 1, 4))
        stds = [np.sqrt(((emb[labels == c] - cents[c]) ** 2).mean(0).sum()) for c in range(4)]
        stats.append((max(stds), min_d, min_d / (max(stds) + 1e-6)))
    max_std, min_d, ratio = np.median(np.array(stats), axis=0)
    assert max_std > 0.05 and min_d > 0.8 and ratio > 1.5


def test_module_fit_transform_and_cosine():
    x = workloads.three_centres(200, 10)
    emb = umapers.fit_transform(x, n_neighbors=10, init="random")
    assert emb.shape == (200, 2) and np.all(np.isfinite(emb))
    emb_c = Umap(n_neighbors=10, metric="cosine").fit_transform(x)
    assert np.all(np.isfinite(emb_c))


def test_knn_diagnostics_reports_recall():
    x = workloads.reference_synthetic(180, 8)
    d = Umap(n_neighbors=10, approx_knn_candidates=28, approx_knn_iters=8).knn_diagnostics(x)
    assert 0.0 <= d["min_recall"] <= d["worst_decile_recall"] <= d["mean_recall"] <= 1.0
    assert d["per_row_recall"].shape == (180,)


def test_full_fit_quality_matches_oracle_mixture(orc):
    x = workloads.isotropic_mixture(5000, 64, 10, 4.0, seed=7)
    g = Umap(n_neighbors=15, n_epochs=200, ann_mode="exact").fit_transform(x)
    o = orc.fit_transform(x, n_neighbors=15, n_epochs=200, use_approximate_knn=0)
    qg, qo = diagnostics.quality(x, g), diagnostics.quality(x, o)
    print("gpu", qg, "oracle", qo)
    assert abs(qg["trustworthiness"] - qo["trustworthiness"]) <= 0.005
    assert abs(qg["knn_preservation"] - qo["knn_preservation"]) <= 0.005 or \
        qg["knn_preservation"] > qo["knn_preservation"]


def test_device_rows_are_validated_before_the_fit():
    """transform_rows / validate_data's finiteness check (lib.rs:2113-2138)
    on rows already on the device: the first non-finite row is named, for an
    aligned array whose last elements do not fill a 16-byte vector and for an
    array that starts off a 16-byte boundary."""
    import torch

    from umapers_b200 import _lib

    lib = _lib.load()
    n, d = 1001, 3
    x = np.random.default_rng(0).normal(size=(n, d)).astype(np.float32)
    out = torch.empty((n, 2), dtype=torch.float32, device="cuda")
    m = Umap(n_neighbors=10, n_epochs=10, ann_mode="exact")

    def fit_device(ptr):
        _lib.check(lib.umapb_fit_transform_device(m._core._handle, ptr, n, d, out.data_ptr(),
                                                  None, None))

    bad = x.copy()
    bad[1000, 2] = np.nan  # element 3002: past the last whole float4
    xd = torch.from_numpy(bad).cuda()
    assert xd.data_ptr() % 16 == 0
    with pytest.raises(ValueError, match="non-finite value at row 1000"):
        fit_device(xd.data_ptr())
    bad = x.copy()
    bad[517, 1] = np.inf
    bad[900, 0] = np.nan
    flat = torch.zeros(n * d + 1, dtype=torch.float32, device="cuda")
    flat[1:] = torch.from_numpy(bad.ravel()).cuda()
    assert (flat.data_ptr() + 4) % 16 != 0
    with pytest.raises(ValueError, match="non-finite value at row 517"):
        fit_device(flat.data_ptr() + 4)
    fit_device(torch.from_numpy(x).cuda().data_ptr())  # finite rows fit
    assert torch.isfinite(out).all()


def test_repeated_fits_reuse_their_device_buffers():
    """A model's second and later fits of the same rows make no new device
    allocation: released buffers are kept per stream and exact size and
    handed back, so the memory pool's mapped and handed-out bytes stay as the
    second fit left them."""
    import ctypes

    from umapers_b200 import _lib

    lib = _lib.load()
    x = workloads.anisotropic_mixture(60_000, 32, 20, seed=9)
    m = Umap(n_neighbors=15, n_epochs=50, ann_mode="exact")

    def pool():
        reserved, used = ctypes.c_int64(0), ctypes.c_int64(0)
        _lib.check(lib.umapb_pool_bytes(ctypes.byref(reserved), ctypes.byref(used)))
        return reserved.value, used.value

    m.fit(x)
    m.fit(x)
    after_second = pool()
    for _ in range(3):
        m.fit(x)
        assert pool() == after_second
    assert np.all(np.isfinite(m.embedding_))


def test_device_fit_profile_outputs_do_not_change_the_fit():
    """umapb_fit_transform_device with and without timings / info: the same
    embedding (1,000 rows run the deterministic one-CTA layout), and the
    profile fields are filled only when asked for."""
    import ctypes

    import torch

    from umapers_b200 import _lib

    lib = _lib.load()
    n, d = 1000, 16
    x = np.random.default_rng(3).normal(size=(n, d)).astype(np.float32)
    xd = torch.from_numpy(x).cuda()
    m = Umap(n_neighbors=15, n_epochs=50, ann_mode="exact", random_seed=9)
    plain = torch.empty((n, 2), dtype=torch.float32, device="cuda")
    prof = torch.empty_like(plain)
    _lib.check(lib.umapb_fit_transform_device(m._core._handle, xd.data_ptr(), n, d,
                                              plain.data_ptr(), None, None))
    t, info = _lib.Timings(), _lib.FitInfo()
    _lib.check(lib.umapb_fit_transform_device(m._core._handle, xd.data_ptr(), n, d,
                                              prof.data_ptr(), ctypes.byref(t), ctypes.byref(info)))
    assert torch.equal(plain, prof)
    assert info.n_samples == n and info.n_edges > 0 and info.sgd_edge_samples > 0
    assert t.total_sec > 0.0 and t.knn_sec > 0.0
