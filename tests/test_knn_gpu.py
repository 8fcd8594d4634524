"""Exact kNN on the GPU against the oracle: indices bit-exact (ties to the
lower index) and FP32 distances bit-exact, for the scalar (dim < 64) and
AVX2 lane (dim >= 64) summation orders, euclidean and cosine, self joins
and query-to-reference searches."""
import numpy as np
import pytest

from umapers_b200 import workloads
from tests import gpu_util as gu

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n,d,k", [(1000, 32, 15), (2000, 64, 15), (1500, 100, 10), (700, 8, 5),
                                   (513, 200, 30)])
def test_plain_knn_bit_exact(orc, n, d, k):
    x = workloads.isotropic_mixture(n, d, 6, 3.0, seed=n + d)
    gi, gd, _ = gu.knn_exact(x, k, backend="plain")
    oi, od = orc.exact_knn(x, k)
    np.testing.assert_array_equal(gi, oi)
    np.testing.assert_array_equal(gd, od)


def test_plain_knn_cosine_bit_exact(orc):
    x = workloads.isotropic_mixture(1200, 72, 5, 2.0, seed=9)
    x[5] = 0.0  # zero-norm row: distance 1 to everything, 0 to itself
    gi, gd, _ = gu.knn_exact(x, 12, metric="cosine", backend="plain")
    oi, od = orc.exact_knn(x, 12, metric="cosine")
    np.testing.assert_array_equal(gi, oi)
    np.testing.assert_array_equal(gd, od)


def test_knn_query_bit_exact(orc):
    fit, q = workloads.transform_mixture(n_fit=3000, n_query=700, d=64, n_comp=8)
    gi, gd = gu.knn_query(q, fit, 15)
    oi, od = orc.knn_query(q, fit, 15)
    np.testing.assert_array_equal(gi, oi)
    np.testing.assert_array_equal(gd, od)


def test_duplicate_rows_resolve_to_lower_index(orc):
    x = workloads.gaussian(400, 16, seed=5)
    x[100:110] = x[50]
    gi, gd, _ = gu.knn_exact(x, 12)
    oi, od = orc.exact_knn(x, 12)
    np.testing.assert_array_equal(gi, oi)
    assert list(gi[105, :11]) == [50] + list(range(100, 110))


def test_mixture_20000x192_sampled_rows_bit_exact(orc):
    x = workloads.isotropic_mixture(20_000, 192, 10, 4.0, seed=7)
    gi, gd, _ = gu.knn_exact(x, 15, backend="plain")
    rows = np.random.default_rng(7).choice(20_000, 200, replace=False)
    oi, od = orc.exact_knn_rows(x, rows, 15)
    np.testing.assert_array_equal(gi[rows], oi)
    np.testing.assert_array_equal(gd[rows], od)


@pytest.mark.parametrize("n,d,k", [(300, 32, 15), (2000, 64, 15), (1500, 100, 10), (3000, 16, 30),
                                   (700, 8, 5), (2500, 130, 15)])
def test_tensor_knn_matches_plain_and_oracle(orc, n, d, k):
    x = workloads.isotropic_mixture(n, d, 6, 3.0, seed=n + 3 * d)
    ti, td, fb = gu.knn_exact(x, k, backend="tensor")
    oi, od = orc.exact_knn(x, k)
    np.testing.assert_array_equal(ti, oi)
    np.testing.assert_array_equal(td, od)
    assert fb <= n // 20  # certification keeps almost every row on the tensor path


def test_tensor_knn_duplicates_and_ties(orc):
    x = workloads.gaussian(600, 64, seed=5)
    # 101 identical rows: each of the two 32-entry lists a row keeps per
    # column half sees more than 32 of them, so no list can hold all the ties
    x[100:200] = x[50]
    ti, td, fb = gu.knn_exact(x, 15, backend="tensor")
    oi, od = orc.exact_knn(x, 15)
    np.testing.assert_array_equal(ti, oi)
    np.testing.assert_array_equal(td, od)
    assert fb >= 101  # rows whose ties exceed the shortlists go to the plain kernel


def test_tensor_knn_ties_that_fit_the_lists_are_certified(orc):
    x = workloads.gaussian(600, 64, seed=5)
    x[100:140] = x[50]  # 41 ties, split 13 / 28 over the two column halves
    ti, td, fb = gu.knn_exact(x, 15, backend="tensor")
    oi, od = orc.exact_knn(x, 15)
    np.testing.assert_array_equal(ti, oi)
    np.testing.assert_array_equal(td, od)
    assert fb < 41


def test_tensor_knn_query_to_reference(orc):
    fit, q = workloads.transform_mixture(n_fit=5000, n_query=900, d=128, n_comp=10)
    ti, td = gu.knn_query(q, fit, 15, backend="tensor")
    oi, od = orc.knn_query(q, fit, 15)
    np.testing.assert_array_equal(ti, oi)
    np.testing.assert_array_equal(td, od)


def test_tensor_knn_mixture_20000x192_sampled_rows(orc):
    x = workloads.isotropic_mixture(20_000, 192, 10, 4.0, seed=7)
    ti, td, fb = gu.knn_exact(x, 15, backend="tensor")
    pi, pd, _ = gu.knn_exact(x, 15, backend="plain")
    np.testing.assert_array_equal(ti, pi)
    np.testing.assert_array_equal(td, pd)
    rows = np.random.default_rng(1).choice(20_000, 200, replace=False)
    oi, od = orc.exact_knn_rows(x, rows, 15)
    np.testing.assert_array_equal(ti[rows], oi)
    assert fb <= 1000


def test_tensor_knn_in_cell_order_matches_plain():
    # at least one wave of query groups: the rows are regrouped by nearest
    # pivot and each group starts at its own cell; the result keeps original
    # row numbers and the lower-index tie rule, duplicates across cells included
    x = workloads.anisotropic_mixture(60_000, 64, 50, seed=3)
    x[59_000:59_020] = x[17]
    x[123] = x[40_000]
    ti, td, fb = gu.knn_exact(x, 15, backend="tensor")
    pi, pd, _ = gu.knn_exact(x, 15, backend="plain")
    np.testing.assert_array_equal(ti, pi)
    np.testing.assert_array_equal(td, pd)
    assert fb <= 600


def test_tensor_knn_large_query_set_matches_plain():
    # a query set of more query tiles than SMs (no candidate splits) runs
    # without the cell order, its candidate walks staggered by unit; 19,000
    # rows leave the last query tile partial
    x = workloads.anisotropic_mixture(30_000, 64, 20, seed=4)
    q = workloads.anisotropic_mixture(19_000, 64, 20, seed=5)
    ti, td = gu.knn_query(q, x, 15, backend="tensor")
    pi, pd = gu.knn_query(q, x, 15, backend="plain")
    np.testing.assert_array_equal(ti, pi)
    np.testing.assert_array_equal(td, pd)


def test_tensor_knn_1m_x_64_sampled_rows(orc):
    x = workloads.anisotropic_mixture(1_000_000, 64, 50, seed=11)
    ti, td, fb = gu.knn_exact(x, 15, backend="tensor")
    rows = np.random.default_rng(11).choice(1_000_000, 64, replace=False)
    oi, od = orc.exact_knn_rows(x, rows, 15)
    np.testing.assert_array_equal(ti[rows], oi)
    np.testing.assert_array_equal(td[rows], od)
    # size-independent properties on every row: self first at 0, sorted rows
    assert np.all(ti[:, 0] == np.arange(1_000_000)) and np.all(td[:, 0] == 0.0)
    assert np.all(np.diff(td, axis=1) >= 0)
    print("fallback rows", fb)
    assert fb <= 10_000


@pytest.mark.parametrize("n,d,k", [(2000, 64, 15), (1500, 40, 10), (2500, 130, 30)])
def test_tensor_knn_cosine_bit_exact(orc, n, d, k):
    # unit-normalised FP16 tiles, bound on 1 - cos, re-rank with the
    # reference's cosine_distance_with_norms (clamp, zero-norm rules)
    x = workloads.isotropic_mixture(n, d, 6, 3.0, seed=n + 5 * d)
    x[7] = 0.0  # zero query row: recomputed on the plain path
    x[11] = -x[12]  # opposite rows: cosine distance 2
    ti, td, fb = gu.knn_exact(x, k, metric="cosine", backend="tensor")
    oi, od = orc.exact_knn(x, k, metric="cosine")
    np.testing.assert_array_equal(ti, oi)
    np.testing.assert_array_equal(td, od)
    assert 1 <= fb <= n // 20


def test_tensor_knn_cosine_20000x192(orc):
    x = workloads.isotropic_mixture(20_000, 192, 10, 4.0, seed=7)
    ti, td, _ = gu.knn_exact(x, 15, metric="cosine", backend="tensor")
    pi, pd, _ = gu.knn_exact(x, 15, metric="cosine", backend="plain")
    np.testing.assert_array_equal(ti, pi)
    np.testing.assert_array_equal(td, pd)
    rows = np.random.default_rng(3).choice(20_000, 100, replace=False)
    oi, od = orc.exact_knn_rows(x, rows, 15, metric="cosine")
    np.testing.assert_array_equal(ti[rows], oi)
    np.testing.assert_array_equal(td[rows], od)


def test_tensor_knn_cosine_query_to_reference(orc):
    fit, q = workloads.transform_mixture(n_fit=4000, n_query=600, d=96, n_comp=10)
    ti, td = gu.knn_query(q, fit, 15, metric="cosine", backend="tensor")
    oi, od = orc.knn_query(q, fit, 15, metric="cosine")
    np.testing.assert_array_equal(ti, oi)
    np.testing.assert_array_equal(td, od)


def test_tensor_knn_second_pass_rows_stay_exact():
    # Well-separated clusters far from the origin: |x|^2 is about 16 d while
    # neighbour distances are about 2 d, so the one-term FP16 bound leaves
    # some rows uncertified after the first pass (four lists per row).  They
    # are re-run with twice the lists; the result equals the plain FP32 path
    # on every row.
    from umapers import Umap

    x = workloads.isotropic_mixture(30_000, 128, 20, 4.0, seed=5)
    prof = Umap(n_neighbors=15, n_epochs=20, ann_mode="exact", knn_backend="tensor",
                init="random").profile_fit_transform(x)
    assert prof["knn_backend"] == "tensor"
    print("second pass rows", prof["knn_second_pass_rows"], "plain rows", prof["knn_fallback_rows"])
    assert prof["knn_second_pass_rows"] > 0
    assert prof["knn_fallback_rows"] <= prof["knn_second_pass_rows"] // 10
    ti, td, _ = gu.knn_exact(x, 15, backend="tensor")
    pi, pd, _ = gu.knn_exact(x, 15, backend="plain")
    np.testing.assert_array_equal(ti, pi)
    np.testing.assert_array_equal(td, pd)


@pytest.mark.parametrize("d", [500, 640, 784, 1100])
def test_tensor_knn_wide_rows(orc, d):
    # 128-candidate tiles (two lists per row) once 256-candidate tiles no
    # longer fit shared memory beside the resident query tile; past that the
    # query tile streams through the ring with the candidate tiles
    x = workloads.isotropic_mixture(3000, d, 8, 1.0, seed=d)
    ti, td, fb = gu.knn_exact(x, 12, backend="tensor")
    rows = np.random.default_rng(d).choice(3000, 80, replace=False)
    oi, od = orc.exact_knn_rows(x, rows, 12)
    np.testing.assert_array_equal(ti[rows], oi)
    np.testing.assert_array_equal(td[rows], od)
    pi, pd, _ = gu.knn_exact(x, 12, backend="plain")
    np.testing.assert_array_equal(ti, pi)
    np.testing.assert_array_equal(td, pd)


@pytest.mark.parametrize("metric", ["euclidean", "cosine"])
def test_tensor_knn_k50_bit_exact(orc, metric):
    # 64-entry re-rank lists: k up to 62 stays on the tensor path
    x = workloads.isotropic_mixture(2000, 64, 6, 3.0, seed=50)
    ti, td, fb = gu.knn_exact(x, 50, metric=metric, backend="tensor")
    oi, od = orc.exact_knn(x, 50, metric=metric)
    np.testing.assert_array_equal(ti, oi)
    np.testing.assert_array_equal(td, od)
    assert fb <= 100


def test_tensor_knn_k50_mixture_20000x192(orc):
    x = workloads.isotropic_mixture(20_000, 192, 10, 4.0, seed=7)
    ti, td, _ = gu.knn_exact(x, 50, backend="tensor")
    pi, pd, _ = gu.knn_exact(x, 50, backend="plain")
    np.testing.assert_array_equal(ti, pi)
    np.testing.assert_array_equal(td, pd)
    rows = np.random.default_rng(50).choice(20_000, 60, replace=False)
    oi, od = orc.exact_knn_rows(x, rows, 50)
    np.testing.assert_array_equal(ti[rows], oi)


def test_tensor_knn_pixel_like_rows_784(orc):
    # non-negative rows far from the origin (pixel intensities 0..255, 784
    # columns): the scaled one-term bound is wide against neighbour gaps, the
    # second pass settles the rest; every row equals the plain path
    rng = np.random.default_rng(784)
    base = rng.uniform(0, 255, size=(10, 784))
    lab = rng.integers(0, 10, size=6000)
    x = np.clip(base[lab] + rng.normal(0, 40, size=(6000, 784)), 0, 255).astype(np.float32)
    ti, td, _ = gu.knn_exact(x, 15, backend="tensor")
    pi, pd, _ = gu.knn_exact(x, 15, backend="plain")
    np.testing.assert_array_equal(ti, pi)
    np.testing.assert_array_equal(td, pd)
    rows = rng.choice(6000, 40, replace=False)
    oi, od = orc.exact_knn_rows(x, rows, 15)
    np.testing.assert_array_equal(ti[rows], oi)
