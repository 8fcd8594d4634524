"""The allocation-free kNN entry point (umapb_knn_exact_noalloc).

It serves callers that cannot allocate device memory, such as a host that
hands all HBM to its own arena, or code that runs where the CUDA allocator
may not be called.  Its scratch is one static 64 MiB device array.  The test
drives it through the C ABI on caller-owned device buffers and checks two
calls in a row against umapb_knn_exact: same indices and the same FP32
distances (exact kNN is index work, so the tolerance is zero).  It also
covers rows recomputed on the plain path (ties beyond the shortlists), a
smaller call of another shape right after a larger one in the same array,
and the rejection of an input above the static limit with a clear error.  This
file sorts last so that a run stopping at the first failure has run every
other test first.
"""
import ctypes

import numpy as np
import pytest

from umapers_b200 import _lib, workloads

pytestmark = pytest.mark.gpu


def _stream_ptr(torch):
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def test_noalloc_knn_matches_the_allocating_entry_point_twice():
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    n, d, k = 20_000, 64, 15
    x = workloads.isotropic_mixture(n, d, 10, 4.0, seed=3)
    ref_i = np.empty((n, k), np.int64)
    ref_d = np.empty((n, k), np.float32)
    _lib.check(lib.umapb_knn_exact(x.ctypes.data, n, d, k, 0, 1, ref_i.ctypes.data,
                                   ref_d.ctypes.data, None))
    xd = torch.from_numpy(x).cuda()
    for _ in range(2):
        out_i = torch.full((n, k), -1, dtype=torch.int32, device="cuda")
        out_d = torch.full((n, k), float("nan"), dtype=torch.float32, device="cuda")
        _lib.check(lib.umapb_knn_exact_noalloc(xd.data_ptr(), n, d, k, out_i.data_ptr(),
                                               out_d.data_ptr(), _stream_ptr(torch)))
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out_i.cpu().numpy().astype(np.int64), ref_i)
        np.testing.assert_array_equal(out_d.cpu().numpy(), ref_d)


def _noalloc(lib, torch, xd, k):
    n, d = xd.shape
    out_i = torch.full((n, k), -1, dtype=torch.int32, device="cuda")
    out_d = torch.full((n, k), float("nan"), dtype=torch.float32, device="cuda")
    _lib.check(lib.umapb_knn_exact_noalloc(xd.data_ptr(), n, d, k, out_i.data_ptr(),
                                           out_d.data_ptr(), _stream_ptr(torch)))
    torch.cuda.synchronize()
    return out_i.cpu().numpy().astype(np.int64), out_d.cpu().numpy()


def _exact(lib, x, k):
    n, d = x.shape
    ref_i = np.empty((n, k), np.int64)
    ref_d = np.empty((n, k), np.float32)
    _lib.check(lib.umapb_knn_exact(x.ctypes.data, n, d, k, 0, 1, ref_i.ctypes.data,
                                   ref_d.ctypes.data, None))
    return ref_i, ref_d


def test_noalloc_knn_recomputes_uncertified_rows_and_reuses_the_array():
    """Rows whose ties overflow the shortlists take the plain path over the
    caller's rows; then a smaller call with other n_rows and n_cols follows
    the larger one in the same array, which still holds that call's data."""
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    x = workloads.gaussian(6000, 64, seed=5)
    x[100:300] = x[50]  # 201 identical rows: more than any list can hold
    ref_i, ref_d = _exact(lib, x, 15)
    got_i, got_d = _noalloc(lib, torch, torch.from_numpy(x).cuda(), 15)
    np.testing.assert_array_equal(got_i, ref_i)
    np.testing.assert_array_equal(got_d, ref_d)
    assert list(got_i[150, :15]) == [50] + list(range(100, 114))
    small = workloads.isotropic_mixture(3000, 40, 6, 3.0, seed=8)
    ref_i, ref_d = _exact(lib, small, 10)
    got_i, got_d = _noalloc(lib, torch, torch.from_numpy(small).cuda(), 10)
    np.testing.assert_array_equal(got_i, ref_i)
    np.testing.assert_array_equal(got_d, ref_d)


def test_noalloc_knn_rejects_inputs_above_its_static_limit():
    torch = pytest.importorskip("torch")
    lib = _lib.load()
    n, d, k = 100_000, 64, 15
    xd = torch.zeros((n, d), dtype=torch.float32, device="cuda")
    out_i = torch.empty((n, k), dtype=torch.int32, device="cuda")
    out_d = torch.empty((n, k), dtype=torch.float32, device="cuda")
    st = lib.umapb_knn_exact_noalloc(xd.data_ptr(), n, d, k, out_i.data_ptr(), out_d.data_ptr(),
                                     _stream_ptr(torch))
    assert st == _lib.ERR_INVALID_PARAMETER
    msg = _lib.last_error()
    assert "static limit" in msg and "rows" in msg
