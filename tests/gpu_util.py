"""Helpers for the GPU parity tests: thin calls into libumapb200.so."""
import ctypes

import numpy as np

from umapers_b200 import _lib

METRIC = {"euclidean": 0, "cosine": 2}
BACKEND = {"auto": 0, "tensor": 1, "plain": 2}


def _p(a):
    return None if a is None else a.ctypes.data


def knn_exact(x, k, metric="euclidean", backend="plain"):
    x = np.ascontiguousarray(x, np.float32)
    n, d = x.shape
    idx = np.empty((n, k), np.int64)
    dist = np.empty((n, k), np.float32)
    fb = ctypes.c_int64(0)
    _lib.check(_lib.load().umapb_knn_exact(_p(x), n, d, k, METRIC[metric], BACKEND[backend],
                                           _p(idx), _p(dist), ctypes.byref(fb)))
    return idx, dist, fb.value


def knn_query(q, r, k, metric="euclidean", backend="plain"):
    q = np.ascontiguousarray(q, np.float32)
    r = np.ascontiguousarray(r, np.float32)
    idx = np.empty((q.shape[0], k), np.int64)
    dist = np.empty((q.shape[0], k), np.float32)
    _lib.check(_lib.load().umapb_knn_query(_p(q), q.shape[0], _p(r), r.shape[0], q.shape[1], k,
                                           METRIC[metric], BACKEND[backend], _p(idx), _p(dist)))
    return idx, dist


def nndescent(x, k, candidates, iters, seed, metric="euclidean", stats=None):
    x = np.ascontiguousarray(x, np.float32)
    n, d = x.shape
    idx = np.empty((n, k), np.int64)
    dist = np.empty((n, k), np.float32)
    ran = ctypes.c_int64(0)
    evaluated = ctypes.c_int64(0)
    ksec = ctypes.c_double(0.0)
    _lib.check(_lib.load().umapb_nndescent(_p(x), n, d, k, METRIC[metric], candidates, iters,
                                           seed & 0xFFFFFFFFFFFFFFFF, _p(idx), _p(dist),
                                           ctypes.byref(ran), ctypes.byref(evaluated),
                                           ctypes.byref(ksec)))
    if stats is not None:
        stats["candidates"] = evaluated.value
        stats["kernel_sec"] = ksec.value
    return idx, dist, ran.value


def smooth_knn(dists, k, local_connectivity=1.0, bandwidth=1.0, include_self=True):
    d = np.ascontiguousarray(dists, np.float32)
    n, c = d.shape
    sig = np.empty(n, np.float32)
    rho = np.empty(n, np.float32)
    _lib.check(_lib.load().umapb_smooth_knn_dist(_p(d), n, c, k, local_connectivity, bandwidth,
                                                 int(include_self), _p(sig), _p(rho)))
    return sig, rho


def fuzzy_graph(idx, dist, mix=1.0, local_connectivity=1.0, n_epochs=0):
    idx = np.ascontiguousarray(idx, np.int64)
    dist = np.ascontiguousarray(dist, np.float32)
    n, k = idx.shape
    cap = 2 * n * k
    h = np.empty(cap, np.int32)
    t = np.empty(cap, np.int32)
    w = np.empty(cap, np.float32)
    sig = np.empty(n, np.float32)
    rho = np.empty(n, np.float32)
    ne = ctypes.c_int64(0)
    _lib.check(_lib.load().umapb_fuzzy_graph(_p(idx), _p(dist), n, k, mix, local_connectivity,
                                             n_epochs, _p(h), _p(t), _p(w), cap, ctypes.byref(ne),
                                             _p(sig), _p(rho)))
    m = ne.value
    return h[:m].copy(), t[:m].copy(), w[:m].copy(), sig, rho


def fuzzy_graph_supervised(idx, dist, labels, target_weight, mix=1.0, local_connectivity=1.0,
                           n_epochs=0):
    idx = np.ascontiguousarray(idx, np.int64)
    dist = np.ascontiguousarray(dist, np.float32)
    labels = np.ascontiguousarray(labels, np.int64)
    n, k = idx.shape
    cap = 2 * n * k
    h = np.empty(cap, np.int32)
    t = np.empty(cap, np.int32)
    w = np.empty(cap, np.float32)
    ne = ctypes.c_int64(0)
    _lib.check(_lib.load().umapb_fuzzy_graph_supervised(
        _p(idx), _p(dist), n, k, mix, local_connectivity, n_epochs, _p(labels), target_weight,
        _p(h), _p(t), _p(w), cap, ctypes.byref(ne)))
    m = ne.value
    return h[:m].copy(), t[:m].copy(), w[:m].copy()


def spectral_init(x, h, t, w, dim, seed):
    x = np.ascontiguousarray(x, np.float32)
    n, d = x.shape
    h = np.ascontiguousarray(h, np.int32)
    t = np.ascontiguousarray(t, np.int32)
    w = np.ascontiguousarray(w, np.float32)
    out = np.empty((n, dim), np.float32)
    used = ctypes.c_int32(0)
    _lib.check(_lib.load().umapb_spectral_init(_p(x), n, d, _p(h), _p(t), _p(w), h.shape[0], dim,
                                               seed, _p(out), ctypes.byref(used)))
    return out, bool(used.value)


def optimize_layout(emb, h, t, w, n_epochs, a, b, lr=1.0, neg_rate=5, repulsion=1.0, seed=0):
    emb = np.array(emb, dtype=np.float32, copy=True, order="C")
    h = np.ascontiguousarray(h, np.int32)
    t = np.ascontiguousarray(t, np.int32)
    w = np.ascontiguousarray(w, np.float32)
    n, dim = emb.shape
    _lib.check(_lib.load().umapb_optimize_layout(_p(emb), n, dim, _p(h), _p(t), _p(w), h.shape[0],
                                                 n_epochs, a, b, lr, neg_rate, repulsion,
                                                 seed & 0xFFFFFFFFFFFFFFFF))
    return emb


def linear_fit_r2(src, dst):
    """R^2 of the best affine map src -> dst (subspace agreement up to rotation)."""
    A = np.hstack([src.astype(np.float64), np.ones((src.shape[0], 1))])
    coef, *_ = np.linalg.lstsq(A, dst.astype(np.float64), rcond=None)
    res = dst - A @ coef
    return 1.0 - (res ** 2).sum() / ((dst - dst.mean(0)) ** 2).sum()
