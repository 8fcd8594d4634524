"""Categorical supervision on the GPU against the oracle.

apply_categorical_target_intersection (rust_umap/src/lib.rs:3694-3760) is
pinned bit for bit: the GPU's supervised graph equals the oracle's
restatement applied to the GPU's own unsupervised graph, for several target
weights, with unlabelled (-1) rows, before and after prune.  The fit follows
the reference's supervised tests (lib.rs:7337-7460): weight 0 leaves the
graph unchanged, a positive weight changes the embedding, -1 labels are
accepted, mismatched label lengths are rejected.  The embedding is compared
with the oracle's pipeline on the same graph by trustworthiness.
"""
import numpy as np
import pytest

from umapers import Umap, fit_transform
from umapers_b200 import diagnostics, workloads
from tests import gpu_util as gu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case(orc):
    x = workloads.isotropic_mixture(3000, 16, 6, 3.0, seed=31)
    idx, dist = orc.exact_knn(x, 15)
    rng = np.random.default_rng(5)
    labels = rng.integers(0, 3, size=x.shape[0]).astype(np.int64)
    labels[::7] = -1
    return x, idx, dist, labels


@pytest.mark.parametrize("weight", [0.3, 0.6, 1.0])
@pytest.mark.parametrize("n_epochs", [0, 200])
def test_supervised_graph_is_bit_exact(orc, case, weight, n_epochs):
    _, idx, dist, labels = case
    uh, ut, uw, _, _ = gu.fuzzy_graph(idx, dist)
    gh, gt, gw = gu.fuzzy_graph_supervised(idx, dist, labels, weight, n_epochs=n_epochs)
    oh, ot, ow = orc.categorical_intersection(uh, ut, uw, labels, weight, n_epochs=n_epochs)
    np.testing.assert_array_equal(gh, oh)
    np.testing.assert_array_equal(gt, ot)
    np.testing.assert_array_equal(gw.view(np.uint32), ow.view(np.uint32))
    if weight == 1.0:
        # exp(-1e12) is 0: no edge joins two different labels
        lh, lt = labels[gh], labels[gt]
        assert np.all((lh == lt) | (lh == -1) | (lt == -1))


def test_weight_zero_leaves_the_graph_unchanged(case):
    _, idx, dist, labels = case
    uh, ut, uw, _, _ = gu.fuzzy_graph(idx, dist, n_epochs=200)
    gh, gt, gw = gu.fuzzy_graph_supervised(idx, dist, labels, 0.0, n_epochs=200)
    np.testing.assert_array_equal(gh, uh)
    np.testing.assert_array_equal(gt, ut)
    np.testing.assert_array_equal(gw, uw)


def _label_separation(emb, labels):
    """Distance between the two label centroids over the mean within-label spread."""
    c = [emb[labels == g].mean(0) for g in (0, 1)]
    spread = np.mean([np.linalg.norm(emb[labels == g] - c[g], axis=1).mean() for g in (0, 1)])
    return float(np.linalg.norm(c[0] - c[1]) / spread)


def test_supervision_separates_arbitrary_labels():
    # categorical_supervision_changes_embedding_when_weight_positive
    # (lib.rs:7368-7398), with labels that do not follow the data
    x = workloads.gaussian(2000, 12, seed=9)
    labels = np.random.default_rng(2).integers(0, 2, size=2000).astype(np.int64)
    base = Umap(n_neighbors=15, n_epochs=200, random_seed=3).fit_transform(x)
    sup = Umap(n_neighbors=15, n_epochs=200, random_seed=3, target_metric="categorical",
               target_weight=0.7).fit_transform(x, labels)
    assert np.all(np.isfinite(sup))
    assert not np.array_equal(base, sup)
    s0, s1 = _label_separation(base, labels), _label_separation(sup, labels)
    print("label separation unsupervised", s0, "supervised", s1)
    assert s0 < 0.3 and s1 > 2.0


def test_supervised_fit_matches_the_oracle_pipeline(orc, case):
    x, idx, dist, labels = case
    emb = Umap(n_neighbors=15, n_epochs=200, random_seed=4, target_metric="categorical",
               target_weight=0.5).fit_transform(x, labels)
    uh, ut, uw, _, _ = orc.fuzzy_graph(idx, dist)
    h, t, w = orc.categorical_intersection(uh, ut, uw, labels, 0.5, n_epochs=200)
    init, _, _ = orc.spectral_init(x, h, t, w, 2, 4)
    a, b = orc.find_ab_params(1.0, 0.1)
    o_emb, _ = orc.optimize_layout(init, h, t, w, 200, a, b, seed=4)
    qg = diagnostics.quality(x, emb, sample=None)
    qo = diagnostics.quality(x, o_emb, sample=None)
    print("gpu", qg, "oracle", qo)
    assert abs(qg["trustworthiness"] - qo["trustworthiness"]) <= 0.01
    sg = _label_separation(emb, (labels == 0).astype(np.int64))
    so = _label_separation(o_emb, (labels == 0).astype(np.int64))
    assert abs(sg - so) <= 0.25 * max(so, 1.0)


def test_supervised_surface(case):
    x, _, _, labels = case
    # categorical_supervision_accepts_unlabeled_minus_one (lib.rs:7420-7460)
    m = Umap(n_neighbors=10, n_epochs=50, target_metric="categorical", target_weight=0.5)
    assert m.fit(x, labels) is m
    assert m.embedding_.shape == (3000, 2) and np.all(np.isfinite(m.embedding_))
    out = np.empty((3000, 2), np.float32)
    assert m.fit_transform(x, labels, out=out) is out
    assert np.all(np.isfinite(out))
    # transform of new rows after a supervised fit uses the fitted embedding
    q = m.transform(x[:50])
    assert q.shape == (50, 2) and np.all(np.isfinite(q))
    emb = fit_transform(x, labels, n_neighbors=10, n_epochs=50, target_metric="categorical")
    assert emb.shape == (3000, 2)
    # y without target_metric is ignored, as in the reference facade
    a = Umap(n_neighbors=10, n_epochs=50).fit_transform(x, labels)
    assert a.shape == (3000, 2)
    # categorical_supervision_rejects_label_length_mismatch (lib.rs:7400-7418)
    with pytest.raises(ValueError, match="target label length"):
        Umap(n_neighbors=10, target_metric="categorical").fit(x, labels[:-1])
