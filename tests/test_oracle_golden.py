"""The CPU oracle against the reference's own known-answer tests (golden
vectors transcribed by tests/golden/make_pins.py) and its internal
consistency properties.  No GPU needed."""
import numpy as np
import pytest

from umapers_b200 import workloads


def test_find_ab_params_bits_match_reference(orc, pins):
    # rust_umap/src/lib.rs:5781-5795
    for case in pins["find_ab_params"]:
        a_bits, b_bits = orc.find_ab_bits(case["spread"], case["min_dist"])
        assert (a_bits, b_bits) == (case["a_bits"], case["b_bits"]), case


@pytest.mark.parametrize("case_idx", [0, 1])
def test_smooth_knn_self_and_non_self_layouts_agree(orc, pins, case_idx):
    # rust_umap/src/lib.rs:6975-7020
    case = pins["smooth_knn_cases"][case_idx]
    s1, r1 = orc.smooth_knn(np.array(case["with_self"]), case["k"], include_self=True)
    s2, r2 = orc.smooth_knn(np.array(case["without_self"]), case["k"], include_self=False)
    assert np.all(np.abs(s1 - s2) <= case["sigma_tol"])
    assert np.all(np.abs(r1 - r2) <= case["rho_tol"])


def test_laplacian_from_edges_matches_dense_affinity(orc, pins):
    # rust_umap/src/lib.rs:7457-7538
    lap = pins["laplacian_edges"]
    e = np.array(lap["edges"])
    l1, l2 = orc.laplacians(lap["n"], e[:, 0], e[:, 1], e[:, 2])
    assert np.max(np.abs(l1 - l2)) < lap["tol"]


def test_smooth_knn_fp32_tracks_fp64(orc):
    rng = np.random.default_rng(0)
    d = np.sort(rng.gamma(2.0, 1.0, size=(500, 15)).astype(np.float32), axis=1)
    d[:, 0] = 0.0
    s32, r32 = orc.smooth_knn(d, 15.0)
    s64, r64 = orc.smooth_knn_f64(d, 15.0)
    np.testing.assert_array_equal(r32, r64.astype(np.float32))
    # the bisection stops at |psum - target| < 1e-5, so sigma agrees to that scale
    assert np.median(np.abs(s32 - s64) / s64) < 1e-5
    assert np.max(np.abs(s32 - s64) / s64) < 1e-3


def test_exact_knn_orders_by_distance_then_index(orc):
    x = workloads.gaussian(300, 70, seed=3)
    x[10] = x[20]  # an exact duplicate pair: ties resolve to the lower index
    idx, dist = orc.exact_knn(x, 8)
    rows = np.arange(300)
    assert np.all(idx[rows != 20, 0] == rows[rows != 20])
    assert idx[20, 0] == 10 and idx[20, 1] == 20 and dist[20, 0] == 0.0 and dist[20, 1] == 0.0
    assert idx[10, 0] == 10 and idx[10, 1] == 20
    assert np.all(np.diff(dist, axis=1) >= 0)
    # same sets as a float64 brute force wherever no near-tie straddles the cut
    d64 = ((x[:, None, :].astype(np.float64) - x[None, :, :]) ** 2).sum(-1)
    order = np.argsort(d64, axis=1, kind="stable")[:, :8]
    agree = np.mean([set(order[i]) == set(idx[i]) for i in range(300)])
    assert agree > 0.99


def test_squared_distance_uses_lane_order(orc):
    # dim >= 64: eight lane sums added in order, then the scalar tail
    rng = np.random.default_rng(1)
    x = rng.normal(size=67).astype(np.float32) * 1000
    y = rng.normal(size=67).astype(np.float32)
    lanes = np.zeros(8, np.float32)
    for i in range(0, 64, 8):
        df = x[i:i + 8] - y[i:i + 8]
        lanes = (lanes + df * df).astype(np.float32)
    s = np.float32(lanes[0])
    for v in lanes[1:]:
        s = np.float32(s + v)
    for i in range(64, 67):
        df = np.float32(x[i] - y[i])
        s = np.float32(s + np.float32(df * df))
    assert orc.squared_distance(x, y) == s


def test_nndescent_recall_reference_threshold(orc):
    # rust_umap/src/lib.rs:6733-6748: recall >= 0.70 excluding self
    x = workloads.reference_synthetic(240, 8)
    ex, _ = orc.exact_knn(x, 12)
    ap, _, _ = orc.nndescent(x, 12, 30, 8, 0x123456789ABCDEF0)
    hits = sum(len(set(ex[i, 1:]) & set(ap[i, 1:])) for i in range(240))
    assert hits / (240 * 11) >= 0.70


def test_oracle_fit_is_deterministic(orc):
    # rust_umap/src/lib.rs:6172-6190
    x = workloads.reference_synthetic(60, 6)
    kw = dict(n_neighbors=10, n_epochs=40, init="random", random_seed=1234)
    a = orc.fit_transform(x, **kw)
    b = orc.fit_transform(x, **kw)
    np.testing.assert_array_equal(a, b)
    assert np.all(np.isfinite(a))


def test_transform_sgd_thread_count_deterministic(orc, pins):
    # rust_umap/src/lib.rs:6193-6236
    p = pins["transform_determinism"]
    base = np.array([[np.sin(i * 0.07), np.cos(i * 0.11)] for i in range(p["n_tail"])], np.float32)
    init = np.array([[np.sin(i * 0.03), np.cos(i * 0.05)] for i in range(p["n_heads"])], np.float32)
    heads = np.repeat(np.arange(p["n_heads"]), 12)
    tails = np.array([(h * 7 + o * 11) % p["n_tail"] for h in range(p["n_heads"]) for o in range(12)])
    w = np.array([1.0 - o * 0.04 for _ in range(p["n_heads"]) for o in range(12)], np.float32)
    args = (init, base, heads, tails, w, p["n_epochs"], p["a"], p["b"], p["alpha"], p["neg_rate"],
            p["repulsion"], p["seed"])
    orc.set_threads(1)
    one = orc.optimize_layout_transform(*args)
    orc.set_threads(4)
    four = orc.optimize_layout_transform(*args)
    orc.set_threads(orc.max_threads())
    np.testing.assert_array_equal(one, four)


def test_spectral_disconnected_beats_random(orc):
    # rust_umap/src/lib.rs:7541-7570
    x, labels = workloads.disconnected_components(4, 60)
    idx, dist = orc.exact_knn(x, 10)
    h, t, w, _, _ = orc.fuzzy_graph(idx, dist)
    spec, used, ncomp = orc.spectral_init(x, h, t, w, 2, 42)
    assert used and ncomp == 4
    rnd = orc.random_init(x.shape[0], 2, 42)

    def ratio(e):
        cents = np.stack([e[labels == c].mean(0) for c in range(4)])
        sep = min(np.linalg.norm(cents[i] - cents[j]) for i in range(4) for j in range(i + 1, 4))
        std = max(np.sqrt(((e[labels == c] - cents[c]) ** 2).mean(0).sum()) for c in range(4))
        return sep / (std + 1e-6)

    assert ratio(spec) > ratio(rnd) * 1.2


def test_densmap_lambda_zero_matches_standard(orc):
    # densmap_lambda_zero_matches_standard_umap (rust_umap/src/lib.rs:6077-6104):
    # synthetic_data(72, 7), k=8, 30 epochs, random init, seed 141, exact kNN
    from umapers_b200 import workloads

    x = workloads.reference_synthetic(72, 7)
    kw = dict(n_neighbors=8, n_epochs=30, init=0, random_seed=141, use_approximate_knn=0)
    std = orc.fit_transform(x, **kw)
    dens, _, _ = orc.fit_transform_dens(x, densmap=1, dens_lambda=0.0, **kw)
    assert np.array_equal(std, dens)


def test_output_dens_radii_are_finite(orc):
    # output_dens_returns_finite_radii (rust_umap/src/lib.rs:6106-6136)
    from umapers_b200 import workloads

    x = workloads.reference_synthetic(64, 6)
    emb, r0, r1 = orc.fit_transform_dens(x, n_neighbors=8, n_epochs=30, init=0, random_seed=143,
                                         use_approximate_knn=0, output_dens=1)
    assert emb.shape == (64, 2) and r0.shape == (64,) and r1.shape == (64,)
    assert np.all(np.isfinite(r0)) and np.all(np.isfinite(r1))


def test_local_radii_follow_the_reference_rule(orc):
    # mean over non-self neighbours of ln(max(d, 0) + var_shift) (lib.rs:5057-5082)
    idx = np.array([[0, 1, 2], [1, 0, 2], [2, 5, 6]], np.int64)
    dist = np.array([[0.0, 1.0, 2.0], [0.0, 1.0, 3.0], [0.0, 0.5, 0.25]], np.float32)
    r = orc.local_radii(idx, dist, 0.1)
    f = np.float32
    expect = [(np.log(f(1.1)) + np.log(f(2.1))) / 2, (np.log(f(1.1)) + np.log(f(3.1))) / 2,
              (np.log(f(0.6)) + np.log(f(0.35))) / 2]
    np.testing.assert_allclose(r, np.array(expect, np.float32), rtol=1e-6)


def _sparse_like_data(n, dim):
    """sparse_like_data (rust_umap/src/lib.rs:5767-5778) in float32."""
    data = np.zeros((n, dim), np.float32)
    f = np.float32
    for i in range(n):
        for t in range(5):
            col = (i * 17 + t * 13 + (i % 3) * 7) % dim
            data[i, col] = f(f(f(i + 1) * f(t + 2)) * f(0.017)) + f(f(col) * f(1e-4))
    return data


def test_sparse_knn_matches_the_dense_knn(orc):
    # sparse_csr_knn_matches_dense_euclidean (rust_umap/src/lib.rs:6376-6394)
    sp = pytest.importorskip("scipy.sparse")
    x = _sparse_like_data(42, 61)
    csr = sp.csr_matrix(x)
    si, sd = orc.csr_knn(csr, 12, "euclidean")
    di, dd = orc.exact_knn(x, 12, "euclidean")
    np.testing.assert_array_equal(si, di)
    assert np.abs(sd - dd).max() <= 1e-5


def test_sparse_knn_follows_the_reference_formulas(orc):
    # sparse.rs:220-244, 368-384, 605-626 on a hand-made matrix: an empty row,
    # a duplicate row, a row with no shared column
    sp = pytest.importorskip("scipy.sparse")
    dense = np.array([[1.0, 0.0, 2.0, 0.0],
                      [0.0, 0.0, 0.0, 0.0],
                      [1.0, 0.0, 2.0, 0.0],
                      [0.0, 3.0, 0.0, -1.0]], np.float32)
    csr = sp.csr_matrix(dense)
    idx, dist = orc.csr_knn(csr, 4, "euclidean")
    f = np.float32
    # row 0: itself 0, its duplicate 0 (by the formula: 5 + 5 - 2 * 5), the
    # empty row sqrt(5), row 3 sqrt(5 + 10)
    np.testing.assert_array_equal(idx[0], [0, 2, 1, 3])
    np.testing.assert_array_equal(dist[0], [0.0, 0.0, np.sqrt(f(5.0)), np.sqrt(f(15.0))])
    idx, dist = orc.csr_knn(csr, 4, "cosine")
    # the empty row: 0 to itself, 1 to every non-empty row (index order)
    np.testing.assert_array_equal(idx[1], [1, 0, 2, 3])
    np.testing.assert_array_equal(dist[1], [0.0, 1.0, 1.0, 1.0])
    # row 3 shares no column with rows 0 / 2: cosine 1
    assert dist[3][1] == f(1.0)


def test_categorical_intersection_pins_the_reference_test(orc):
    # categorical_target_intersection_modulates_existing_feature_edges
    # (rust_umap/src/lib.rs:7256-7335): the same ten data edges, labels
    # [0, 0, 1, 1], target weight 0.6
    pairs = [(0, 1, 0.8), (1, 0, 0.8), (0, 2, 0.7), (2, 0, 0.7), (1, 2, 0.4), (2, 1, 0.4),
             (2, 3, 0.8), (3, 2, 0.8), (0, 3, 0.6), (3, 0, 0.6)]
    h = np.array([p[0] for p in pairs], np.int32)
    t = np.array([p[1] for p in pairs], np.int32)
    w = np.array([p[2] for p in pairs], np.float32)
    labels = np.array([0, 0, 1, 1], np.int64)
    oh, ot, ow = orc.categorical_intersection(h, t, w, labels, 0.6)
    assert set(zip(oh.tolist(), ot.tolist())) <= set(zip(h.tolist(), t.tolist()))
    weight = {(a, b): c for a, b, c in zip(oh.tolist(), ot.tolist(), ow.tolist())}
    wt = lambda a, b: weight.get((a, b), 0.0)  # noqa: E731
    assert wt(0, 1) > wt(0, 2) and wt(1, 0) > wt(1, 2)
    assert wt(2, 3) > wt(2, 0) and wt(3, 2) > wt(3, 0)
    # the same steps written out in float32: scale, divide by the head's
    # largest weight, fuzzy union with mix 1
    far = np.float32(np.exp(-np.float32(2.5) / (np.float32(1.0) - np.float32(0.6))))
    scaled = {(a, b): np.float32(c) * (np.float32(1.0) if labels[a] == labels[b] else far)
              for a, b, c in pairs}
    row_max = {i: max(v for (a, _), v in scaled.items() if a == i) for i in range(4)}
    directed = {(a, b): np.float32(v / row_max[a]) for (a, b), v in scaled.items()}
    for (a, b), v in directed.items():
        u = directed[(b, a)]
        expect = np.float32(np.float32(v + u) - np.float32(v * u))
        assert np.float32(wt(a, b)) == expect, (a, b)
    # weight 0 leaves the graph unchanged; weight 1 drops the cross-label edges
    zh, zt, zw = orc.categorical_intersection(h, t, w, labels, 0.0)
    np.testing.assert_array_equal(zw, w)
    ah, at, aw = orc.categorical_intersection(h, t, w, labels, 1.0)
    assert all(labels[a] == labels[b] for a, b in zip(ah.tolist(), at.tolist()))
    # an unlabelled end scales by exp(-1), far less than a label mismatch
    lab_u = np.array([0, -1, 1, 1], np.int64)
    uh, ut, uw = orc.categorical_intersection(h, t, w, lab_u, 0.6)
    uwt = {(a, b): c for a, b, c in zip(uh.tolist(), ut.tolist(), uw.tolist())}
    assert uwt[(1, 2)] > 100 * wt(1, 2)


def test_inverse_transform_restatement_basics(orc):
    # inverse_transform_workflow (rust_umap/src/lib.rs:6271-6293) on the
    # oracle: shape, finiteness, and an embedded point that is a fitted point
    # (distance 0 <= 1e-6) maps back to that row exactly (lib.rs:1890, 4856)
    x = workloads.reference_synthetic(140, 6)
    idx, dist = orc.exact_knn(x, 15)
    _, _, _, sig, rho = orc.fuzzy_graph(idx, dist)
    rng = np.random.default_rng(0)
    emb = (x[:, :2] + 0.01 * rng.normal(size=(140, 2))).astype(np.float32)
    a, b = orc.find_ab_params(1.0, 0.1)
    rec = orc.inverse_transform(x, emb, sig, rho, emb[130:], n_neighbors=15, n_epochs=90, a=a, b=b)
    assert rec.shape == (10, 6) and np.all(np.isfinite(rec))
    np.testing.assert_array_equal(rec, x[130:])
    # points between fitted points land near the local linear model's prediction
    mid = ((emb[:10] + emb[10:20]) / 2).astype(np.float32)
    rm = orc.inverse_transform(x, emb, sig, rho, mid, n_neighbors=15, n_epochs=90, a=a, b=b)
    assert np.all(np.isfinite(rm))
    assert np.mean(np.linalg.norm(rm - (x[:10] + x[10:20]) / 2, axis=1)) < \
        np.mean(np.linalg.norm(x - x.mean(0), axis=1))
