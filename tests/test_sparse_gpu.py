"""CSR sparse input on the GPU against the CPU oracle.

The exact sparse kNN is pinned bit for bit against the oracle's restatement
of sparse::exact_nearest_neighbors / exact_nearest_neighbors_sparse_query
(rust_umap/src/sparse.rs:605-657): indices and FP32 distances, euclidean and
cosine, on inputs with negative values, empty rows, duplicate rows and rows
of equal norm, over more than one 2048-row tile.  The fit and transform follow
the reference's sparse tests (rust_umap/src/lib.rs:6376-6660, 7568-7740):
sparse kNN equals the dense kNN of the same matrix, sparse and dense queries
of a sparse model transform alike, sparse queries need a sparse model, and a
disconnected sparse graph still gets a spectral layout.
"""
import ctypes

import numpy as np
import pytest

from umapers import Umap, fit_transform
from umapers_b200 import _lib, diagnostics, workloads

sp = pytest.importorskip("scipy.sparse")
pytestmark = pytest.mark.gpu


def _matrix(n, d, density, seed, empty_rows=(), dup_pairs=(), lognormal=False):
    rng = np.random.default_rng(seed)
    m = sp.random(n, d, density=density, format="csr", dtype=np.float32,
                  random_state=np.random.RandomState(seed))
    if lognormal:
        m.data = rng.lognormal(0.0, 1.0, size=m.data.shape).astype(np.float32)
    else:
        m.data = rng.normal(size=m.data.shape).astype(np.float32)
    m = m.tolil()
    for r in empty_rows:
        m.rows[r] = []
        m.data[r] = []
    for a, b in dup_pairs:
        m.rows[b] = list(m.rows[a])
        m.data[b] = list(m.data[a])
    m = m.tocsr()
    m.sort_indices()
    return m


def _parts(m):
    return (np.ascontiguousarray(m.indptr, np.int64), np.ascontiguousarray(m.indices, np.int64),
            np.ascontiguousarray(m.data, np.float32))


def _gpu_knn(m, k, metric):
    lib = _lib.load()
    ip, ix, dv = _parts(m)
    n, d = m.shape
    idx = np.empty((n, k), np.int64)
    dist = np.empty((n, k), np.float32)
    code = {"euclidean": 0, "cosine": 2}[metric]
    _lib.check(lib.umapb_knn_csr(ip.ctypes.data, ix.ctypes.data, dv.ctypes.data, n, d, k, code,
                                 idx.ctypes.data, dist.ctypes.data))
    return idx, dist


def _gpu_knn_query(q, r, k, metric):
    lib = _lib.load()
    qp, qi, qd = _parts(q)
    rp, ri, rd = _parts(r)
    idx = np.empty((q.shape[0], k), np.int64)
    dist = np.empty((q.shape[0], k), np.float32)
    code = {"euclidean": 0, "cosine": 2}[metric]
    _lib.check(lib.umapb_knn_csr_query(qp.ctypes.data, qi.ctypes.data, qd.ctypes.data, q.shape[0],
                                       rp.ctypes.data, ri.ctypes.data, rd.ctypes.data, r.shape[0],
                                       q.shape[1], k, code, idx.ctypes.data, dist.ctypes.data))
    return idx, dist


@pytest.mark.parametrize("metric", ["euclidean", "cosine"])
@pytest.mark.parametrize("k", [5, 15, 30])
def test_sparse_knn_is_bit_exact(orc, metric, k):
    m = _matrix(9000, 300, 0.03, seed=11, empty_rows=(3, 4000, 8999),
                dup_pairs=((10, 20), (5000, 7), (8000, 8001)))
    gi, gd = _gpu_knn(m, k, metric)
    oi, od = orc.csr_knn(m, k, metric)
    np.testing.assert_array_equal(gi, oi)
    np.testing.assert_array_equal(gd.view(np.uint32), od.view(np.uint32))


@pytest.mark.parametrize("metric", ["euclidean", "cosine"])
def test_sparse_query_knn_is_bit_exact(orc, metric):
    r = _matrix(6000, 500, 0.02, seed=3, empty_rows=(17,), lognormal=True)
    q = _matrix(700, 500, 0.02, seed=4, empty_rows=(0, 699), lognormal=True)
    gi, gd = _gpu_knn_query(q, r, 15, metric)
    oi, od = orc.csr_knn_query(q, r, 15, metric)
    np.testing.assert_array_equal(gi, oi)
    np.testing.assert_array_equal(gd.view(np.uint32), od.view(np.uint32))


def test_sparse_knn_matches_dense_knn(orc):
    # sparse_csr_knn_matches_dense_euclidean (rust_umap/src/lib.rs:6376-6394)
    m = _matrix(2000, 64, 0.2, seed=5)
    gi, gd = _gpu_knn(m, 15, "euclidean")
    di, dd = orc.exact_knn(m.toarray(), 15)
    assert (gi == di).mean() > 0.999
    np.testing.assert_allclose(gd, dd, rtol=1e-5, atol=1e-5)


@pytest.fixture(scope="module")
def clusters():
    """Five groups of rows on disjoint column blocks."""
    rng = np.random.default_rng(9)
    blocks = []
    for g in range(5):
        b = sp.random(600, 40, density=0.3, format="csr", dtype=np.float32,
                      random_state=np.random.RandomState(g))
        b.data = (rng.lognormal(0.0, 0.5, size=b.data.shape) + 2.0 * g).astype(np.float32)
        blocks.append(sp.hstack([sp.csr_matrix((600, 40 * g)), b,
                                 sp.csr_matrix((600, 40 * (4 - g)))]).tocsr())
    x = sp.vstack(blocks).tocsr()
    x.sort_indices()
    return x


def test_sparse_fit_matches_the_oracle_pipeline(orc, clusters):
    x = clusters
    emb = Umap(n_neighbors=15, n_epochs=200, random_seed=4, metric="cosine").fit_transform(x)
    assert emb.shape == (3000, 2) and np.all(np.isfinite(emb))
    idx, dist = orc.csr_knn(x, 15, "cosine")
    h, t, w, _, _ = orc.fuzzy_graph(idx, dist, n_epochs=200)
    init, _, _ = orc.spectral_init(x.toarray(), h, t, w, 2, 4)
    a, b = orc.find_ab_params(1.0, 0.1)
    o_emb, _ = orc.optimize_layout(init, h, t, w, 200, a, b, seed=4)
    dense = x.toarray()
    qg = diagnostics.quality(dense, emb, sample=None)
    qo = diagnostics.quality(dense, o_emb, sample=None)
    print("gpu", qg, "oracle", qo)
    assert abs(qg["trustworthiness"] - qo["trustworthiness"]) <= 0.01


def test_sparse_and_dense_queries_transform_alike(clusters):
    # sparse_csr_query_transform_matches_dense_query_transform (lib.rs:6429-6472)
    x = clusters
    m = Umap(n_neighbors=12, n_epochs=100, random_seed=2).fit(x)
    q = x[::7]
    a = m.transform(q)
    b = m.transform(q.toarray())
    np.testing.assert_array_equal(a, b)
    assert np.all(np.isfinite(a))
    out = np.empty_like(a)
    assert m.transform(q, out=out) is out
    np.testing.assert_array_equal(out, a)


def test_sparse_transform_contracts(clusters):
    x = clusters
    dense_model = Umap(n_neighbors=10, n_epochs=50).fit(x.toarray())
    with pytest.raises(ValueError, match="supported only for sparse-fitted models"):
        dense_model.transform(x[:5])
    m = Umap(n_neighbors=10, n_epochs=50).fit(x)
    with pytest.raises(ValueError, match="feature mismatch"):
        m.transform(x[:5, :100])
    assert m.transform(x[:0]).shape == (0, 2)
    with pytest.raises(ValueError, match="needs a model fitted on dense rows"):
        m.fit_surrogate(epochs=1)


def _separation(emb, labels, n_comp):
    """min_centroid_distance, max_component_std and separation_ratio of the
    reference tests (rust_umap/src/lib.rs:5890-5959)."""
    cents = np.stack([emb[labels == c].mean(0) for c in range(n_comp)])
    min_d = min(np.linalg.norm(cents[i] - cents[j])
                for i in range(n_comp) for j in range(i + 1, n_comp))
    max_std = max(float(np.sqrt((emb[labels == c].std(0) ** 2).sum())) for c in range(n_comp))
    return min_d, max_std, min_d / (max_std + 1e-6)


def test_disconnected_sparse_graph_gets_a_spectral_layout():
    # sparse_spectral_init_handles_disconnected_components (lib.rs:7697-7740)
    x, labels = workloads.disconnected_components(4, 60)
    csr = sp.csr_matrix(x)
    csr.eliminate_zeros()
    emb = Umap(n_neighbors=10, n_components=2, n_epochs=60, metric="euclidean", init="spectral",
               random_seed=42, ann_mode="exact").fit_transform(csr)
    assert np.all(np.isfinite(emb))
    min_d, max_std, ratio = _separation(emb, labels, 4)
    print("min centroid distance", min_d, "max std", max_std, "ratio", ratio)
    assert max_std > 0.05 and min_d > 0.8 and ratio > 1.1


def test_module_fit_transform_and_formats(clusters):
    x = clusters
    dense = x.toarray()
    trust = []
    for data in (x, x.tocsc(), x.tocoo()):
        emb = fit_transform(data, n_neighbors=10, n_epochs=50, random_seed=3)
        assert emb.shape == (3000, 2) and np.all(np.isfinite(emb))
        trust.append(diagnostics.quality(dense, emb, sample=None)["trustworthiness"])
    print("trust by input format", trust)
    # the same CSR rows whatever the format; Hogwild runs differ only in update order
    assert max(trust) - min(trust) <= 0.02
    m = Umap(n_neighbors=10, n_epochs=50).fit(x)
    assert m.n_features_in_ == 200 and m.n_samples_fit_ == 3000


def _gpu_nndescent_csr(m, k, metric, candidates, iters, seed=99):
    ip, ix, dv = _parts(m)
    n, d = m.shape
    idx = np.empty((n, k), np.int64)
    dist = np.empty((n, k), np.float32)
    ran, ev = ctypes.c_int64(0), ctypes.c_int64(0)
    ksec = ctypes.c_double(0.0)
    _lib.check(_lib.load().umapb_nndescent_csr(
        ip.ctypes.data, ix.ctypes.data, dv.ctypes.data, n, d, k, {"euclidean": 0, "cosine": 2}[metric],
        candidates, iters, seed, idx.ctypes.data, dist.ctypes.data, ctypes.byref(ran),
        ctypes.byref(ev), ctypes.byref(ksec)))
    return idx, dist, ran.value, ev.value


def _topics(n, d, n_topics, per_row, seed):
    """Text-like CSR rows: each row draws most of its columns from its topic's
    block of preferred columns, the rest anywhere; LogNormal(0, 1) values."""
    rng = np.random.default_rng(seed)
    pref = [rng.choice(d, 60, replace=False) for _ in range(n_topics)]
    rows, cols = [], []
    for r in range(n):
        t = rng.integers(n_topics)
        c = np.concatenate([rng.choice(pref[t], int(per_row * 0.8), replace=False),
                            rng.integers(0, d, per_row - int(per_row * 0.8))])
        c = np.unique(c)
        rows.append(np.full(c.shape[0], r))
        cols.append(c)
    rows, cols = np.concatenate(rows), np.concatenate(cols)
    vals = rng.lognormal(0.0, 1.0, size=rows.shape[0]).astype(np.float32)
    m = sp.csr_matrix((vals, (rows, cols)), shape=(n, d))
    m.sort_indices()
    return m


@pytest.mark.parametrize("metric", ["cosine", "euclidean"])
def test_sparse_nndescent_recall_against_exact(orc, metric):
    """NN-descent on CSR rows (the reference's candidate rule, the exact
    sparse kNN's distances): every listed distance equals the exact sparse
    distance of that pair, lists are sorted with self first, and recall@15
    against the exact sparse kNN (itself bit-exact with the oracle) matches
    the recall of the oracle's NN-descent on the same rows densified, at the
    reference's default 50 candidates and 14 iterations.  Euclidean distances
    on these rows are hub-dominated (rows with small norms are near to
    everyone), and the reference's algorithm itself reaches about 0.55 there;
    cosine reaches about 0.94."""
    m = _topics(6000, 2000, 20, 20, seed=21)
    k = 15
    ai, ad, ran, ev = _gpu_nndescent_csr(m, k, metric, 50, 14)
    ei, ed = _gpu_knn(m, k, metric)
    assert 1 <= ran <= 14 and ev > 6000 * 50
    assert np.all(ai[:, 0] == np.arange(6000)) and np.all(ad[:, 0] == 0.0)
    assert np.all(np.diff(ad, axis=1) >= 0)
    recall = np.mean([len(set(ai[r]) & set(ei[r])) / k for r in range(6000)])
    x = m.toarray().astype(np.float32)
    oi = orc.nndescent(x, k, 50, 14, 99, metric=metric)[0]
    oe = orc.exact_knn(x, k, metric=metric)[0]
    ref = np.mean([len(set(oi[r]) & set(oe[r])) / k for r in range(6000)])
    print(metric, "recall", recall, "oracle recall", ref, "iterations", ran)
    assert recall >= ref - 0.02
    if metric == "cosine":
        assert recall >= 0.9
    # a pair listed by both has the same FP32 distance
    for r in range(0, 6000, 97):
        common = set(ai[r]) & set(ei[r])
        for j in common:
            assert ad[r][list(ai[r]).index(j)] == ed[r][list(ei[r]).index(j)]


def test_sparse_fit_takes_nndescent_on_explicit_approximate_request():
    m = _topics(3000, 500, 10, 20, seed=4)
    emb = Umap(n_neighbors=15, metric="cosine", n_epochs=50, ann_mode="approximate",
               random_seed=3).fit_transform(m)
    exact = Umap(n_neighbors=15, metric="cosine", n_epochs=50, ann_mode="exact",
                 random_seed=3).fit_transform(m)
    dense = m.toarray()
    ta = diagnostics.quality(dense, emb, sample=None)["trustworthiness"]
    te = diagnostics.quality(dense, exact, sample=None)["trustworthiness"]
    print("trust approximate", ta, "exact", te)
    assert np.all(np.isfinite(emb)) and abs(ta - te) <= 0.02
