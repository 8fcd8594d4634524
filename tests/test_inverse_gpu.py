"""inverse_transform on the GPU against the oracle.

inverse_transform_rows (rust_umap/src/lib.rs:1800-1915): kNN of the embedded
queries among the fitted embedding, weights 1 / (1 + a d^(2b)), the local
linear init (init_inverse_points, lib.rs:4838-4935) and the inverse SGD
(optimize_layout_inverse, lib.rs:5547-5645).  An embedded point that is a
fitted point maps back to its row exactly.  Other queries are compared with
the oracle's restatement on the same model (the GPU's embedding, the fit's
sigmas and rhos) by reconstruction error: the reference's SGD draws its
negatives from one sequential generator, the GPU from one stream per query.
"""
import numpy as np
import pytest

from umapers import Umap
from umapers_b200 import workloads

pytestmark = pytest.mark.gpu


def test_inverse_transform_workflow():
    # inverse_transform_workflow (lib.rs:6271-6293)
    x = workloads.reference_synthetic(140, 6)
    m = Umap(n_neighbors=15, n_components=2, n_epochs=90, init="spectral", random_seed=11)
    emb = m.fit_transform(x)
    rec = m.inverse_transform(emb[130:])
    assert rec.shape == (10, 6) and np.all(np.isfinite(rec))
    # each query is a fitted point: its first neighbour is itself at distance 0
    first = [int(np.argmin(np.linalg.norm(emb - q, axis=1))) for q in emb[130:]]
    np.testing.assert_array_equal(rec, x[first])
    out = np.empty((10, 6), np.float32)
    assert m.inverse_transform(emb[130:], out=out) is out
    np.testing.assert_array_equal(out, rec)
    assert m.inverse_transform(np.empty((0, 2), np.float32)).shape == (0, 6)


def _recon_error(rec, truth):
    return float(np.mean(np.linalg.norm(rec - truth, axis=1)))


def test_inverse_transform_matches_the_oracle(orc):
    fit, held = workloads.transform_mixture(n_fit=4000, n_query=300, d=24, n_comp=6)
    m = Umap(n_neighbors=15, n_epochs=200, random_seed=7)
    emb = m.fit_transform(fit)
    q = m.transform(held)
    rec = m.inverse_transform(q)
    assert rec.shape == (300, 24) and np.all(np.isfinite(rec))
    idx, dist = orc.exact_knn(fit, 15)
    _, _, _, sig, rho = orc.fuzzy_graph(idx, dist)
    a, b = orc.find_ab_params(1.0, 0.1)
    o_rec = orc.inverse_transform(fit, emb, sig, rho, q, n_neighbors=15, n_epochs=200, a=a, b=b,
                                  seed=42)
    e_gpu, e_orc = _recon_error(rec, held), _recon_error(o_rec, held)
    e_mean = _recon_error(np.broadcast_to(fit.mean(0), held.shape), held)
    print("reconstruction error gpu", e_gpu, "oracle", e_orc, "global mean", e_mean)
    assert e_gpu <= 1.1 * e_orc + 1e-3
    assert e_gpu < 0.8 * e_mean
    # the rows land near the oracle's, far closer than the spread of the data
    assert np.median(np.linalg.norm(rec - o_rec, axis=1)) < 0.5 * e_mean


def test_inverse_transform_contracts():
    x = workloads.reference_synthetic(120, 5)
    with pytest.raises(RuntimeError, match="not fitted"):
        Umap(n_neighbors=10).inverse_transform(np.zeros((1, 2), np.float32))
    m = Umap(n_neighbors=10, n_epochs=30).fit(x)
    with pytest.raises(ValueError, match="embedding dimension mismatch: expected 2, got 3"):
        m.inverse_transform(np.zeros((4, 3), np.float32))
    bad = np.zeros((3, 2), np.float32)
    bad[1, 0] = np.nan
    with pytest.raises(ValueError, match="input contains non-finite value at row 1"):
        m.inverse_transform(bad)
    sp = pytest.importorskip("scipy.sparse")
    ms = Umap(n_neighbors=10, n_epochs=30).fit(sp.csr_matrix(x))
    with pytest.raises(ValueError, match="not supported for sparse-trained models"):
        ms.inverse_transform(np.zeros((2, 2), np.float32))
