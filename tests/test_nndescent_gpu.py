"""NN-descent on the GPU: recall against exact kNN (the reference's
thresholds, rust_umap/src/lib.rs:6733-6764) and against the oracle's own
recall on the same data."""
import numpy as np
import pytest

from umapers_b200 import workloads
from tests import gpu_util as gu

pytestmark = pytest.mark.gpu


def recall(exact, approx):
    hits = sum(len(set(exact[i, 1:]) & set(approx[i, 1:])) for i in range(exact.shape[0]))
    return hits / (exact.shape[0] * (exact.shape[1] - 1))


def test_recall_reference_threshold_euclidean(orc):
    x = workloads.reference_synthetic(240, 8)
    ex, _ = orc.exact_knn(x, 12)
    ap, ad, ran = gu.nndescent(x, 12, 30, 8, 0x123456789ABCDEF0)
    assert recall(ex, ap) >= 0.70
    assert ran >= 1 and np.all(np.diff(ad, axis=1) >= 0)
    assert np.all(ap[:, 0] == np.arange(240))


def test_recall_reference_threshold_cosine(orc):
    x = workloads.reference_synthetic(220, 9)
    ex, _ = orc.exact_knn(x, 10, metric="cosine")
    ap, _, _ = gu.nndescent(x, 10, 28, 8, 0xCAFEBABEDEADC0DE, metric="cosine")
    assert recall(ex, ap) >= 0.65


def test_recall_tracks_oracle_on_mixture(orc):
    x = workloads.anisotropic_mixture(20_000, 64, 20, seed=11)
    rows = np.random.default_rng(0).choice(20_000, 500, replace=False)
    exr, _ = orc.exact_knn_rows(x, rows, 15)
    ap, ad, _ = gu.nndescent(x, 15, 30, 10, 99)
    oa, _, _ = orc.nndescent(x, 15, 30, 10, 99)
    r_gpu = recall(exr, ap[rows])
    r_orc = recall(exr, oa[rows])
    print("recall gpu", r_gpu, "oracle", r_orc)
    assert r_gpu >= r_orc - 0.02
    # distances are exact FP32 distances of the returned pairs
    d_chk = np.sqrt(((x[rows, None, :] - x[ap[rows]]) ** 2).sum(-1))
    np.testing.assert_allclose(ad[rows], d_chk, rtol=1e-5, atol=1e-5)
