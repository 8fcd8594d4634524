"""smooth_knn_dist and the fuzzy union on the GPU against the oracle:
rho bit-exact, sigma and edge weights within 1e-5 relative of the FP32
restatement, and within the bisection's own resolution of the FP64 one."""
import numpy as np
import pytest

from umapers_b200 import workloads
from tests import gpu_util as gu

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def knn(orc):
    x = workloads.isotropic_mixture(4000, 48, 8, 3.0, seed=21)
    idx, dist = orc.exact_knn(x, 15)
    return x, idx, dist


def test_smooth_knn_matches_fp32_oracle(orc, knn):
    _, _, dist = knn
    gs, gr = gu.smooth_knn(dist, 15.0)
    os_, or_ = orc.smooth_knn(dist, 15.0)
    np.testing.assert_array_equal(gr, or_)
    rel = np.abs(gs - os_) / os_
    assert np.mean(rel <= 1e-5) >= 0.999
    assert rel.max() < 1e-3


def test_smooth_knn_tracks_fp64_oracle(orc, knn):
    _, _, dist = knn
    gs, gr = gu.smooth_knn(dist, 15.0)
    s64, r64 = orc.smooth_knn_f64(dist, 15.0)
    np.testing.assert_allclose(gr, r64, rtol=1e-6)
    rel = np.abs(gs - s64) / s64
    assert np.median(rel) < 1e-5 and rel.max() < 1e-3


@pytest.mark.parametrize("case_idx", [0, 1])
def test_smooth_knn_reference_layouts(pins, case_idx):
    case = pins["smooth_knn_cases"][case_idx]
    s1, r1 = gu.smooth_knn(np.array(case["with_self"]), case["k"], include_self=True)
    s2, r2 = gu.smooth_knn(np.array(case["without_self"]), case["k"], include_self=False)
    assert np.all(np.abs(s1 - s2) <= case["sigma_tol"])
    assert np.all(np.abs(r1 - r2) <= case["rho_tol"])


@pytest.mark.parametrize("mix", [1.0, 0.5, 0.0])
def test_fuzzy_union_matches_oracle(orc, knn, mix):
    _, idx, dist = knn
    gh, gt, gw, _, _ = gu.fuzzy_graph(idx, dist, mix=mix)
    oh, ot, ow, _, _ = orc.fuzzy_graph(idx, dist, mix=mix)
    np.testing.assert_array_equal(gh, oh)
    np.testing.assert_array_equal(gt, ot)
    rel = np.abs(gw - ow) / ow
    assert np.mean(rel <= 1e-5) >= 0.999 and rel.max() < 1e-3
    # symmetric: (i, j) and (j, i) carry the same weight
    key = dict(zip(zip(gh.tolist(), gt.tolist()), gw.tolist()))
    assert all(key[(j, i)] == w for (i, j), w in list(key.items())[:2000])


def test_prune_matches_oracle(orc, knn):
    _, idx, dist = knn
    gh, gt, gw, _, _ = gu.fuzzy_graph(idx, dist, n_epochs=200)
    oh, ot, ow, _, _ = orc.fuzzy_graph(idx, dist, n_epochs=200)
    g = set(zip(gh.tolist(), gt.tolist()))
    o = set(zip(oh.tolist(), ot.tolist()))
    assert len(g ^ o) <= max(2, len(o) // 1000)
    assert gw.min() >= gw.max() / 200 * (1 - 1e-6)
