"""transform on the GPU: kNN to the training rows, bipartite membership,
weighted-mean init and per-query SGD (rust_umap/src/lib.rs:1604-1780),
compared with the oracle's transform from the same fitted embedding."""
import numpy as np
import pytest

from umapers import Umap
from umapers_b200 import diagnostics, workloads

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def fitted():
    fit, q = workloads.transform_mixture(n_fit=4000, n_query=1500, d=32, n_comp=8)
    m = Umap(n_neighbors=15, random_seed=3)
    emb = m.fit_transform(fit)
    return m, fit, q, emb


def test_transform_matches_oracle(orc, fitted):
    m, fit, q, emb = fitted
    a, b = m._core.ab_params
    g = m.transform(q)
    o = orc.transform(fit, emb, q, a, b, n_neighbors=15, random_seed=3)
    assert g.shape == (1500, 2) and np.all(np.isfinite(g))
    scale = np.linalg.norm(emb.std(0))
    disp = np.linalg.norm(g - o, axis=1)
    print("median displacement / scale", np.median(disp) / scale)
    assert np.median(disp) < 0.1 * scale
    both_g = np.vstack([fit, q]), np.vstack([emb, g])
    both_o = np.vstack([emb, o])
    tg = diagnostics.quality(both_g[0], both_g[1])["trustworthiness"]
    to = diagnostics.quality(both_g[0], both_o)["trustworthiness"]
    assert abs(tg - to) <= 0.01


def test_transform_of_training_rows_lands_near_fit(fitted):
    m, fit, _, emb = fitted
    g = m.transform(fit[:300])
    scale = np.linalg.norm(emb.std(0))
    assert np.median(np.linalg.norm(g - emb[:300], axis=1)) < 0.2 * scale


def test_transform_out_buffer_empty_and_errors(fitted):
    m, _, q, _ = fitted
    out = np.empty((10, 2), np.float32)
    assert m.transform(q[:10], out=out) is out
    assert m.transform(np.zeros((0, 32), np.float32)).shape == (0, 2)
    with pytest.raises(ValueError, match="feature mismatch"):
        m.transform(np.zeros((3, 31), np.float32))
    bad = q[:5].copy()
    bad[2, 1] = np.inf
    with pytest.raises(ValueError, match="non-finite value at row 2"):
        m.transform(bad)
