"""The learned transform surrogate on the GPU.

1. Gradients: umapb_mlp_grad (tcgen05 forward/backward GEMMs, fused GELU
   epilogues, CUDA-core head and loss) against the CPU FP64 oracle
   (oracle/mlp.py) with bf16 rounding at the same points.
2. Training: the loss falls, held-out rows land near their fitted positions.
3. Gate: rows far from the training distribution go to the plain transform.
4. Gain: on the same queries the surrogate transform is much faster than the
   plain transform at trustworthiness@15 within 0.01 of it.
"""
import ctypes
import time

import numpy as np
import pytest

from oracle import mlp
from umapers import Umap
from umapers_b200 import _lib, diagnostics, workloads

pytestmark = pytest.mark.gpu


def _batch(rng, B, din, hidden, n_out, n_teacher=700, n_neg=5, scale=2.0):
    x = rng.normal(size=(B, din)).astype(np.float32)
    params = mlp.glorot(rng, din, hidden, n_out).astype(np.float32)
    params[mlp.layout(din, hidden, n_out)["b1"][0]:][:hidden] = rng.normal(scale=0.1, size=hidden)
    targets = rng.normal(scale=scale, size=(B, n_out)).astype(np.float32)
    teacher = rng.normal(scale=scale, size=(n_teacher, n_out)).astype(np.float32)
    counts = rng.integers(0, 12, size=B)
    edge_ptr = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
    edge_tail = rng.integers(0, n_teacher, size=edge_ptr[-1]).astype(np.int32)
    edge_weight = rng.uniform(0.05, 1.0, size=edge_ptr[-1]).astype(np.float32)
    neg_tail = rng.integers(0, n_teacher, size=(B, n_neg)).astype(np.int32)
    return x, params, targets, teacher, edge_ptr, edge_tail, edge_weight, neg_tail


def _gpu_grad(x, params, targets, teacher, ep, et, ew, nt, hidden, n_out, a, b, mse_w, edge_w,
              neg_scale, out_shift=None, out_scale=None):
    B, din = x.shape
    mb = _lib.MlpBatch()
    mb.batch, mb.n_features, mb.hidden, mb.n_out = B, din, hidden, n_out
    mb.x, mb.targets, mb.params, mb.teacher = (x.ctypes.data, targets.ctypes.data,
                                               params.ctypes.data, teacher.ctypes.data)
    mb.n_teacher = teacher.shape[0]
    mb.edge_ptr, mb.edge_tail, mb.edge_weight = ep.ctypes.data, et.ctypes.data, ew.ctypes.data
    mb.neg_tail, mb.n_neg = nt.ctypes.data, nt.shape[1]
    mb.a, mb.b, mb.mse_weight, mb.edge_loss_weight, mb.neg_scale = a, b, mse_w, edge_w, neg_scale
    keep = []
    if out_shift is not None:
        keep = [np.ascontiguousarray(out_shift, np.float32), np.ascontiguousarray(out_scale, np.float32)]
        mb.out_shift, mb.out_scale = keep[0].ctypes.data, keep[1].ctypes.data
    grads = np.empty(params.size, np.float32)
    y = np.empty((B, n_out), np.float32)
    loss = ctypes.c_double(0.0)
    _lib.check(_lib.load().umapb_mlp_grad(ctypes.byref(mb), grads.ctypes.data,
                                          ctypes.addressof(loss), y.ctypes.data))
    return grads, loss.value, y


@pytest.mark.parametrize("B,din,hidden,n_out", [(256, 48, 256, 2), (512, 128, 512, 2),
                                                (128, 200, 128, 3)])
def test_mlp_gradients_match_oracle(B, din, hidden, n_out):
    rng = np.random.default_rng(B + din)
    x, params, targets, teacher, ep, et, ew, nt = _batch(rng, B, din, hidden, n_out)
    kw = dict(a=1.577, b=0.895, mse_w=1.0, edge_w=0.5, neg_scale=5.0,
              out_shift=rng.normal(size=n_out), out_scale=rng.uniform(1.0, 4.0, size=n_out))
    g, loss, y = _gpu_grad(x, params, targets, teacher, ep, et, ew, nt, hidden, n_out, **kw)
    og, oloss, oy = mlp.forward_backward(x, targets, params, teacher, ep, et, ew, nt,
                                         hidden=hidden, n_out=n_out, **kw)
    # outputs: FP32 accumulation of bf16 operands against FP64 of the same operands
    assert np.abs(y - oy).max() <= 2e-3 * np.abs(oy).max()
    assert abs(loss - oloss) <= 1e-3 * abs(oloss)
    lay = mlp.layout(din, hidden, n_out)
    for name in ("W1", "b1", "W2", "b2", "W3", "b3"):
        off, size = lay[name]
        gg, oo = g[off:off + size], og[off:off + size]
        rel = np.linalg.norm(gg - oo) / np.linalg.norm(oo)
        worst = np.abs(gg - oo).max() / np.abs(oo).max()
        print(name, "rel", rel, "worst", worst)
        # tolerance: rel. Frobenius 1e-2 and max-abs 2e-2 of the largest entry
        assert rel < 1e-2 and worst < 2e-2, (name, rel, worst)


def test_mlp_gradients_pure_mse_are_tight():
    rng = np.random.default_rng(5)
    x, params, targets, teacher, ep, et, ew, nt = _batch(rng, 256, 64, 256, 2, n_neg=0)
    ep[:] = 0
    kw = dict(a=1.577, b=0.895, mse_w=1.0, edge_w=0.0, neg_scale=5.0)
    g, _, _ = _gpu_grad(x, params, targets, teacher, ep, et[:0], ew[:0], nt, 256, 2, **kw)
    og, _, _ = mlp.forward_backward(x, targets, params, teacher, ep, et[:0], ew[:0], nt,
                                    hidden=256, n_out=2, **kw)
    assert np.linalg.norm(g - og) / np.linalg.norm(og) < 1e-2


@pytest.fixture(scope="module")
def trained():
    fit, query = workloads.transform_mixture(n_fit=40_000, n_query=200_000, d=64)
    m = Umap(n_neighbors=15, random_seed=5, ann_mode="exact")
    emb = m.fit_transform(fit)
    info = m.fit_surrogate(epochs=20, batch_size=1024)
    return m, fit, query, emb, info


def test_training_converges_and_generalises(trained):
    m, fit, _, emb, info = trained
    hist = m._core.surrogate_loss_history()
    print(info)
    assert len(hist) == 20 and hist[-1] < 0.5 * hist[0]
    assert info["n_holdout"] > 0 and info["steps"] == 20 * (info["n_train"] // 1024)
    # the held-out rows were never trained on
    assert info["holdout_within_radius"] > 0.9 and info["holdout_median_error"] < info["radius"]
    assert info["holdout_gated"] < 0.1


def test_gate_sends_out_of_distribution_rows_to_plain(trained):
    """Far rows are gated and recomputed by the plain transform, each as a
    request of its own: with in-distribution rows interleaved into the same
    request (same row positions, same epoch count) the far rows' positions do
    not change, and they stay close to the batch plain transform, which
    differs only through the batch-wide largest weight."""
    m, fit, query, _, _ = trained
    far = query[:500] + 40.0
    out, flags = m._core.transform_surrogate(far, use_fallback=True)
    flags = flags.astype(bool)
    assert flags.mean() > 0.99
    mixed = far.copy()
    mixed[1::2] = query[1000:1250]
    out_m, flags_m = m._core.transform_surrogate(mixed, use_fallback=True)
    flags_m = flags_m.astype(bool)
    both = flags & flags_m
    both[1::2] = False  # other rows there
    assert both[0::2].mean() > 0.99
    np.testing.assert_array_equal(out_m[both], out[both])
    plain = m.transform(far)
    spread = float(np.ptp(m.embedding_, axis=0).max())
    assert np.median(np.abs(out[flags] - plain[flags])) < 0.02 * spread
    _, flags_in = m._core.transform_surrogate(query[:5000], use_fallback=False)
    assert flags_in.mean() < 0.1


def _device_transform(m, q_dev, out_dev, surrogate):
    import torch

    lib = _lib.load()
    n, d = q_dev.shape
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    if surrogate:
        nf = ctypes.c_int64(0)
        _lib.check(lib.umapb_surrogate_transform_device(m._core._handle, q_dev.data_ptr(), n, d, 1,
                                                        out_dev.data_ptr(), None,
                                                        ctypes.byref(nf)))
    else:
        _lib.check(lib.umapb_transform_device(m._core._handle, q_dev.data_ptr(), n, d,
                                              out_dev.data_ptr()))
    torch.cuda.synchronize()
    return time.perf_counter() - t0


def test_surrogate_transform_gain_over_plain(trained):
    """What the trained network gains: the same 200 000 queries through the
    plain transform (kNN to the training rows + SGD refine) and through the
    surrogate with its gate and fallback, device-resident, at equal quality."""
    import torch

    m, fit, query, emb, _ = trained
    q = torch.from_numpy(query).cuda()
    out_p = torch.empty((query.shape[0], 2), dtype=torch.float32, device="cuda")
    out_s = torch.empty_like(out_p)
    for _ in range(2):  # warm-up
        _device_transform(m, q, out_p, False)
        _device_transform(m, q, out_s, True)
    t_plain = min(_device_transform(m, q, out_p, False) for _ in range(3))
    t_sur = min(_device_transform(m, q, out_s, True) for _ in range(3))
    plain, sur = out_p.cpu().numpy(), out_s.cpu().numpy()
    n = 8000
    tp = diagnostics.quality(query[:n], plain[:n])["trustworthiness"]
    ts = diagnostics.quality(query[:n], sur[:n])["trustworthiness"]
    print(f"plain {t_plain:.4f}s surrogate {t_sur:.4f}s ({t_plain / t_sur:.1f}x) "
          f"trust plain {tp:.4f} surrogate {ts:.4f}")
    assert abs(ts - tp) <= 0.01
    assert t_plain / t_sur > 5.0


def test_umap_transform_mode_surrogate_trains_on_fit():
    x = workloads.isotropic_mixture(6000, 32, 6, 4.0, seed=2)
    m = Umap(n_neighbors=15, ann_mode="exact", transform_mode="surrogate",
             surrogate_kwds={"epochs": 3, "batch_size": 1024, "hidden": 256})
    m.fit(x)
    assert m._core.surrogate_ready and m.surrogate_info_["steps"] > 0
    out = m.transform(x[:300])
    assert out.shape == (300, 2) and np.all(np.isfinite(out))
    assert m.transform_fallback_.shape == (300,)
    with pytest.raises(ValueError, match="feature mismatch"):
        m.transform(x[:5, :31])


def test_chunked_host_transform_equals_device_path_and_gated_rows_are_row_local(trained):
    """The host surrogate transform uploads 131,072-row chunks and runs the
    network on each as it lands.  A gated row is transformed as a request of
    its own (its sigma floor, prune threshold and sampling periods from its
    own neighbours) with the random stream of its row in the request, so the
    host path equals the device-resident path bit for bit, and a gated row's
    result does not change when the request holds other rows: the first chunk
    sent alone gives its gated rows the same positions (both requests exceed
    10,000 rows, so both run 30 epochs)."""
    import torch

    m, fit, query, _, _ = trained
    q = np.concatenate([query, query[:400_000] + 0.0])[:600_000].copy()
    q[::97] += 25.0  # out-of-distribution rows in every chunk: gated
    out_h, flags_h = m._core.transform_surrogate(q, use_fallback=True)
    flags_h = flags_h.astype(bool)
    lib = _lib.load()

    def device(rows):
        qd = torch.from_numpy(rows).cuda()
        out_d = torch.empty((rows.shape[0], 2), dtype=torch.float32, device="cuda")
        flags_d = torch.empty(rows.shape[0], dtype=torch.uint8, device="cuda")
        nf = ctypes.c_int64(0)
        _lib.check(lib.umapb_surrogate_transform_device(
            m._core._handle, qd.data_ptr(), rows.shape[0], rows.shape[1], 1, out_d.data_ptr(),
            flags_d.data_ptr(), ctypes.byref(nf)))
        return out_d.cpu().numpy(), flags_d.cpu().numpy().astype(bool), nf.value

    out_d, flags_d, nf = device(q)
    assert flags_h.sum() == nf >= q.shape[0] // 97
    np.testing.assert_array_equal(flags_h, flags_d)
    np.testing.assert_array_equal(out_h, out_d)
    head = q[:131_072].copy()
    out_1, flags_1, nf1 = device(head)
    np.testing.assert_array_equal(flags_1, flags_h[:131_072])
    assert 0 < nf1 < nf
    np.testing.assert_array_equal(out_1[flags_1], out_h[:131_072][flags_1])
    # the network's rows are the same too (row-wise inference)
    np.testing.assert_array_equal(out_1[~flags_1], out_h[:131_072][~flags_1])
