"""Spectral initialisation on the GPU against the oracle: the same
embedding subspace for connected graphs, and component separation for
disconnected ones (rust_umap/src/lib.rs:7541-7694)."""
import numpy as np
import pytest

from umapers_b200 import workloads
from tests import gpu_util as gu

pytestmark = pytest.mark.gpu


def _ratio(e, labels, n):
    cents = np.stack([e[labels == c].mean(0) for c in range(n)])
    sep = min(np.linalg.norm(cents[i] - cents[j]) for i in range(n) for j in range(i + 1, n))
    std = max(np.sqrt(((e[labels == c] - cents[c]) ** 2).mean(0).sum()) for c in range(n))
    return sep / (std + 1e-6)


def test_connected_spectral_matches_oracle_subspace(orc):
    x = workloads.gaussian(2000, 32, seed=4)
    idx, dist = orc.exact_knn(x, 15)
    h, t, w, _, _ = orc.fuzzy_graph(idx, dist, n_epochs=500)
    g, used = gu.spectral_init(x, h, t, w, 2, 42)
    o, oused, ncomp = orc.spectral_init(x, h, t, w, 2, 42)
    assert used and oused and ncomp == 1
    assert np.abs(g).max() == pytest.approx(10.0, abs=1e-2)
    assert gu.linear_fit_r2(o, g) > 0.98 and gu.linear_fit_r2(g, o) > 0.98


def test_disconnected_spectral_beats_random(orc):
    x, labels = workloads.disconnected_components(4, 60)
    idx, dist = orc.exact_knn(x, 10)
    h, t, w, _, _ = orc.fuzzy_graph(idx, dist)
    g, used = gu.spectral_init(x, h, t, w, 2, 42)
    assert used
    rnd = orc.random_init(x.shape[0], 2, 42)
    assert _ratio(g, labels, 4) > _ratio(rnd, labels, 4) * 1.2


def test_large_disconnected_components_stay_structured(orc):
    # components above 128 nodes take the batched iterative path
    x, labels = workloads.disconnected_components(3, 152)
    idx, dist = orc.exact_knn(x, 12)
    h, t, w, _, _ = orc.fuzzy_graph(idx, dist)
    g, used = gu.spectral_init(x, h, t, w, 2, 42)
    assert used and np.all(np.isfinite(g))
    rnd = orc.random_init(x.shape[0], 2, 42)
    assert _ratio(g, labels, 3) > _ratio(rnd, labels, 3) * 1.2


def test_mixture_components_follow_oracle_layout(orc):
    x = workloads.isotropic_mixture(3000, 64, 6, 6.0, seed=8)
    idx, dist = orc.exact_knn(x, 15)
    h, t, w, _, _ = orc.fuzzy_graph(idx, dist, n_epochs=500)
    g, used = gu.spectral_init(x, h, t, w, 2, 7)
    o, oused, ncomp = orc.spectral_init(x, h, t, w, 2, 7)
    assert used and oused and ncomp >= 2
    # component anchors are deterministic (meta layout); within-component
    # coordinates agree up to the eigenvector sign per component
    np.testing.assert_allclose(g.mean(0), o.mean(0), atol=0.5)
