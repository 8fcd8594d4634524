"""ctypes wrapper of the CPU oracle (oracle/umap_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, by __graft_entry__.smoke() as
the checker and by bench.py's CPU-baseline leg.  The product package never
imports it.  The shared object is built by ``make -C oracle`` (g++, OpenMP);
``load()`` builds it when it is missing.
"""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_build" / "libumap_oracle.so"

_f32 = ctypes.c_float
_f64 = ctypes.c_double
_i64 = ctypes.c_int64
_i32 = ctypes.c_int32
_u64 = ctypes.c_uint64
_vp = ctypes.c_void_p

_SIGS = {
    "orc_set_threads": (None, [ctypes.c_int]),
    "orc_max_threads": (ctypes.c_int, []),
    "orc_find_ab_params": (None, [_f32, _f32, ctypes.POINTER(_f32), ctypes.POINTER(_f32)]),
    "orc_squared_distance": (_f32, [_vp, _vp, _i64]),
    "orc_cosine_distance": (_f32, [_vp, _vp, _i64]),
    "orc_exact_knn": (None, [_vp, _i64, _i64, _i64, _i32, _vp, _vp]),
    "orc_exact_knn_rows": (None, [_vp, _i64, _i64, _i64, _i32, _vp, _i64, _vp, _vp]),
    "orc_knn_query": (None, [_vp, _i64, _vp, _i64, _i64, _i64, _i32, _vp, _vp]),
    "orc_csr_knn": (None, [_vp, _vp, _vp, _i64, _i64, _i64, _i32, _vp, _vp]),
    "orc_csr_knn_rows": (None, [_vp, _vp, _vp, _i64, _i64, _vp, _i64, _i64, _i32, _vp, _vp]),
    "orc_csr_knn_query": (
        None, [_vp, _vp, _vp, _i64, _vp, _vp, _vp, _i64, _i64, _i64, _i32, _vp, _vp]),
    "orc_nndescent": (_i64, [_vp, _i64, _i64, _i64, _i32, _i64, _i64, _u64, _vp, _vp]),
    "orc_smooth_knn": (None, [_vp, _i64, _i64, _f32, _f32, _f32, _i32, _vp, _vp]),
    "orc_smooth_knn_f64": (None, [_vp, _i64, _i64, _f64, _f64, _f64, _i32, _vp, _vp]),
    "orc_fuzzy_graph": (
        _i64,
        [_vp, _vp, _i64, _i64, _f32, _f32, _i64, _vp, _vp, _vp, _i64, _vp, _vp],
    ),
    "orc_inverse_transform": (
        _i32, [_vp, _i64, _i64, _vp, _i64, _vp, _vp, _vp, _i64, _i64, _i64, _f32, _f32, _f32,
               _i64, _f32, _u64, _vp]),
    "orc_categorical_intersection": (
        _i64, [_vp, _vp, _vp, _i64, _vp, _i64, _f32, _i64, _vp, _vp, _vp, _i64]),
    "orc_spectral_init": (_i32, [_vp, _i64, _i64, _vp, _vp, _vp, _i64, _i64, _u64, _vp, _vp]),
    "orc_random_init": (None, [_i64, _i64, _u64, _f32, _f32, _vp]),
    "orc_optimize_layout": (
        _f64,
        [_vp, _i64, _i64, _vp, _vp, _vp, _i64, _i64, _f32, _f32, _f32, _i64, _f32, _u64],
    ),
    "orc_fit_transform": (_i32, [_vp, _i64, _i64, _vp, _vp, _vp, _vp, _vp]),
    "orc_fit_transform_dens": (_i32, [_vp, _i64, _i64, _vp, _vp, _vp, _vp]),
    "orc_local_radii": (None, [_vp, _vp, _i64, _i64, _f32, _vp]),
    "orc_transform": (_i32, [_vp, _i64, _vp, _vp, _i64, _i64, _vp, _f32, _f32, _vp]),
    "orc_transform_graph": (_i64, [_vp, _i64, _vp, _vp, _i64, _i64, _vp, _vp, _vp, _vp, _vp,
                                   _vp, _i64, _vp]),
    "orc_optimize_layout_transform": (
        None,
        [_vp, _i64, _i64, _vp, _i64, _vp, _vp, _vp, _i64, _i64, _f32, _f32, _f32, _i64, _f32,
         _u64],
    ),
    "orc_laplacians": (_i32, [_i64, _vp, _vp, _vp, _i64, _vp, _vp]),
    "orc_rng_u64": (None, [_u64, _i64, _vp]),
}

_LIB = None


def load() -> ctypes.CDLL:
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        subprocess.run(["make", "-C", str(HERE)], check=True, capture_output=True)
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _LIB = lib
    return lib


def _p(a):
    return None if a is None else a.ctypes.data


def _f32m(x):
    return np.ascontiguousarray(x, dtype=np.float32)


METRIC = {"euclidean": 0, "cosine": 2}


def set_threads(n: int) -> None:
    load().orc_set_threads(n)


def max_threads() -> int:
    return int(load().orc_max_threads())


def find_ab_params(spread: float, min_dist: float) -> tuple[float, float]:
    a, b = _f32(), _f32()
    load().orc_find_ab_params(spread, min_dist, ctypes.byref(a), ctypes.byref(b))
    return a.value, b.value


def find_ab_bits(spread: float, min_dist: float) -> tuple[int, int]:
    a, b = find_ab_params(spread, min_dist)
    return (int(np.float32(a).view(np.uint32)), int(np.float32(b).view(np.uint32)))


def squared_distance(x, y) -> float:
    x, y = _f32m(x), _f32m(y)
    return float(load().orc_squared_distance(_p(x), _p(y), x.shape[0]))


def exact_knn(x, k: int, metric: str = "euclidean"):
    x = _f32m(x)
    n, d = x.shape
    idx = np.empty((n, k), np.int64)
    dist = np.empty((n, k), np.float32)
    load().orc_exact_knn(_p(x), n, d, k, METRIC[metric], _p(idx), _p(dist))
    return idx, dist


def exact_knn_rows(x, rows, k: int, metric: str = "euclidean"):
    x = _f32m(x)
    rows = np.ascontiguousarray(rows, dtype=np.int64)
    n, d = x.shape
    idx = np.empty((rows.shape[0], k), np.int64)
    dist = np.empty((rows.shape[0], k), np.float32)
    load().orc_exact_knn_rows(_p(x), n, d, k, METRIC[metric], _p(rows), rows.shape[0], _p(idx),
                              _p(dist))
    return idx, dist


def knn_query(q, r, k: int, metric: str = "euclidean"):
    q, r = _f32m(q), _f32m(r)
    idx = np.empty((q.shape[0], k), np.int64)
    dist = np.empty((q.shape[0], k), np.float32)
    load().orc_knn_query(_p(q), q.shape[0], _p(r), r.shape[0], q.shape[1], k, METRIC[metric],
                         _p(idx), _p(dist))
    return idx, dist


def _csr_parts(m):
    """(indptr int64, indices int64, data float32, n_rows, n_cols) of a
    scipy.sparse matrix in canonical CSR form."""
    m = m.tocsr()
    m.sum_duplicates()
    m.sort_indices()
    return (np.ascontiguousarray(m.indptr, np.int64), np.ascontiguousarray(m.indices, np.int64),
            np.ascontiguousarray(m.data, np.float32), m.shape[0], m.shape[1])


def csr_knn(m, k: int, metric: str = "euclidean"):
    """exact_nearest_neighbors of a sparse matrix (sparse.rs:605-626)."""
    ip, ix, dv, n, d = _csr_parts(m)
    idx = np.empty((n, k), np.int64)
    dist = np.empty((n, k), np.float32)
    load().orc_csr_knn(_p(ip), _p(ix), _p(dv), n, d, k, METRIC[metric], _p(idx), _p(dist))
    return idx, dist


def csr_knn_rows(m, rows, k: int, metric: str = "euclidean"):
    """Rows `rows` of exact_nearest_neighbors of a sparse matrix."""
    ip, ix, dv, n, d = _csr_parts(m)
    rows = np.ascontiguousarray(rows, np.int64)
    idx = np.empty((rows.shape[0], k), np.int64)
    dist = np.empty((rows.shape[0], k), np.float32)
    load().orc_csr_knn_rows(_p(ip), _p(ix), _p(dv), n, d, _p(rows), rows.shape[0], k,
                            METRIC[metric], _p(idx), _p(dist))
    return idx, dist


def csr_knn_query(q, r, k: int, metric: str = "euclidean"):
    """exact_nearest_neighbors_sparse_query (sparse.rs:628-657)."""
    qp, qi, qd, nq, d = _csr_parts(q)
    rp, ri, rd, nr, _ = _csr_parts(r)
    idx = np.empty((nq, k), np.int64)
    dist = np.empty((nq, k), np.float32)
    load().orc_csr_knn_query(_p(qp), _p(qi), _p(qd), nq, _p(rp), _p(ri), _p(rd), nr, d, k,
                             METRIC[metric], _p(idx), _p(dist))
    return idx, dist


def nndescent(x, k: int, candidates: int, iters: int, seed: int, metric: str = "euclidean"):
    x = _f32m(x)
    n, d = x.shape
    idx = np.empty((n, k), np.int64)
    dist = np.empty((n, k), np.float32)
    ran = load().orc_nndescent(_p(x), n, d, k, METRIC[metric], candidates, iters,
                               seed & 0xFFFFFFFFFFFFFFFF, _p(idx), _p(dist))
    return idx, dist, int(ran)


def smooth_knn(dists, k: float, local_connectivity: float = 1.0, bandwidth: float = 1.0,
               include_self: bool = True):
    d = _f32m(dists)
    n, kc = d.shape
    sig = np.empty(n, np.float32)
    rho = np.empty(n, np.float32)
    load().orc_smooth_knn(_p(d), n, kc, k, local_connectivity, bandwidth, int(include_self),
                          _p(sig), _p(rho))
    return sig, rho


def smooth_knn_f64(dists, k: float, local_connectivity: float = 1.0, bandwidth: float = 1.0,
                   include_self: bool = True):
    d = _f32m(dists)
    n, kc = d.shape
    sig = np.empty(n, np.float64)
    rho = np.empty(n, np.float64)
    load().orc_smooth_knn_f64(_p(d), n, kc, k, local_connectivity, bandwidth, int(include_self),
                              _p(sig), _p(rho))
    return sig, rho


def fuzzy_graph(idx, dist, mix: float = 1.0, local_connectivity: float = 1.0, n_epochs: int = 0):
    idx = np.ascontiguousarray(idx, dtype=np.int64)
    dist = _f32m(dist)
    n, k = idx.shape
    cap = 2 * n * k
    h = np.empty(cap, np.int32)
    t = np.empty(cap, np.int32)
    w = np.empty(cap, np.float32)
    sig = np.empty(n, np.float32)
    rho = np.empty(n, np.float32)
    ne = load().orc_fuzzy_graph(_p(idx), _p(dist), n, k, mix, local_connectivity, n_epochs,
                                _p(h), _p(t), _p(w), cap, _p(sig), _p(rho))
    return h[:ne].copy(), t[:ne].copy(), w[:ne].copy(), sig, rho


def categorical_intersection(heads, tails, weights, labels, weight: float, n_epochs: int = 0):
    """apply_categorical_target_intersection (lib.rs:3694-3760) of an edge
    list, then prune_edges when n_epochs > 0."""
    heads = np.ascontiguousarray(heads, np.int32)
    tails = np.ascontiguousarray(tails, np.int32)
    weights = _f32m(weights)
    labels = np.ascontiguousarray(labels, np.int64)
    m = heads.shape[0]
    cap = max(m, 1)
    h = np.empty(cap, np.int32)
    t = np.empty(cap, np.int32)
    w = np.empty(cap, np.float32)
    ne = load().orc_categorical_intersection(_p(heads), _p(tails), _p(weights), m, _p(labels),
                                             labels.shape[0], weight, n_epochs, _p(h), _p(t),
                                             _p(w), cap)
    return h[:ne].copy(), t[:ne].copy(), w[:ne].copy()


def inverse_transform(x, emb, sigmas, rhos, query, n_neighbors: int = 15, n_epochs=None,
                      a: float = 1.0, b: float = 1.0, lr: float = 1.0, neg_rate: int = 5,
                      repulsion: float = 1.0, seed: int = 42):
    """inverse_transform_rows (lib.rs:1800-1915) of a model given by its
    rows, embedding and the fit's sigmas / rhos; the SGD seed is the model
    seed ^ 0xD1B54A32D192ED03 as in the reference."""
    x, emb, query = _f32m(x), _f32m(emb), _f32m(query)
    sig = np.ascontiguousarray(sigmas, np.float32)
    rho = np.ascontiguousarray(rhos, np.float32)
    n, d = x.shape
    nq, low = query.shape
    out = np.empty((nq, d), np.float32)
    load().orc_inverse_transform(_p(x), n, d, _p(emb), low, _p(sig), _p(rho), _p(query), nq,
                                 n_neighbors, -1 if n_epochs is None else n_epochs, a, b, lr,
                                 neg_rate, repulsion, (seed ^ 0xD1B54A32D192ED03) & (2**64 - 1),
                                 _p(out))
    return out


def spectral_init(x, heads, tails, weights, dim: int, seed: int):
    x = _f32m(x)
    n, d = x.shape
    heads = np.ascontiguousarray(heads, np.int32)
    tails = np.ascontiguousarray(tails, np.int32)
    weights = _f32m(weights)
    out = np.empty((n, dim), np.float32)
    ncomp = np.zeros(1, np.int64)
    used = load().orc_spectral_init(_p(x), n, d, _p(heads), _p(tails), _p(weights),
                                    heads.shape[0], dim, seed & 0xFFFFFFFFFFFFFFFF, _p(out),
                                    _p(ncomp))
    return out, bool(used), int(ncomp[0])


def random_init(n: int, dim: int, seed: int, low: float = -10.0, high: float = 10.0):
    out = np.empty((n, dim), np.float32)
    load().orc_random_init(n, dim, seed, low, high, _p(out))
    return out


def optimize_layout(emb, heads, tails, weights, n_epochs: int, a: float, b: float,
                    lr: float = 1.0, neg_rate: int = 5, repulsion: float = 1.0, seed: int = 0):
    emb = np.array(emb, dtype=np.float32, copy=True, order="C")
    heads = np.ascontiguousarray(heads, np.int32)
    tails = np.ascontiguousarray(tails, np.int32)
    weights = _f32m(weights)
    n, dim = emb.shape
    samples = load().orc_optimize_layout(_p(emb), n, dim, _p(heads), _p(tails), _p(weights),
                                         heads.shape[0], n_epochs, a, b, lr, neg_rate, repulsion,
                                         seed & 0xFFFFFFFFFFFFFFFF)
    return emb, float(samples)


def _params(**kw):
    """umapb_params with the reference defaults, overridden by kw."""
    import umapers_b200._lib as lib  # struct layout only; no engine call

    p = lib.Params()
    p.n_neighbors, p.n_components, p.n_epochs = 15, 2, -1
    p.metric, p.metric_p = 0, 0.0
    p.learning_rate, p.min_dist, p.spread = 1.0, 0.1, 1.0
    p.local_connectivity, p.set_op_mix_ratio, p.repulsion_strength = 1.0, 1.0, 1.0
    p.negative_sample_rate, p.random_seed, p.init = 5, 42, 1
    p.use_approximate_knn, p.approx_knn_candidates, p.approx_knn_iters = 1, 50, 14
    p.approx_knn_threshold = 4096
    p.densmap, p.dens_lambda, p.dens_frac, p.dens_var_shift, p.output_dens = 0, 2.0, 0.3, 0.1, 0
    p.knn_backend = 0
    for key, val in kw.items():
        if key == "metric" and isinstance(val, str):
            val = METRIC[val]
        if key == "init" and isinstance(val, str):
            val = {"random": 0, "spectral": 1}[val]
        setattr(p, key, val)
    return p


def fit_transform(x, return_stats: bool = False, **kw):
    """Full oracle fit; with return_stats, also per-stage seconds
    (knn, graph, init, sgd), the SGD edge-sample count and the edge count."""
    x = _f32m(x)
    n, d = x.shape
    p = _params(**kw)
    out = np.empty((n, p.n_components), np.float32)
    samples = np.zeros(1, np.float64)
    ne = np.zeros(1, np.int64)
    stages = np.zeros(4, np.float64)
    st = load().orc_fit_transform(_p(x), n, d, ctypes.byref(p), _p(out), _p(samples), _p(ne),
                                  _p(stages))
    if st != 0:
        raise ValueError("oracle does not cover these parameters")
    if return_stats:
        return out, {"knn_sec": stages[0], "graph_sec": stages[1], "init_sec": stages[2],
                     "sgd_sec": stages[3], "edge_samples": float(samples[0]),
                     "n_edges": int(ne[0])}
    return out


def fit_transform_dens(x, **kw):
    """Oracle fit with densMAP / output_dens: (embedding, radii of the input
    neighbourhoods, radii of the embedding neighbourhoods)."""
    x = _f32m(x)
    n, d = x.shape
    p = _params(**kw)
    out = np.empty((n, p.n_components), np.float32)
    r0 = np.empty(n, np.float32)
    r1 = np.empty(n, np.float32)
    if load().orc_fit_transform_dens(_p(x), n, d, ctypes.byref(p), _p(out), _p(r0), _p(r1)):
        raise ValueError("oracle does not cover these parameters")
    return out, r0, r1


def local_radii(idx, dist, var_shift: float = 0.1):
    """local_radii_from_knn (lib.rs:5057-5082) of a kNN table."""
    idx = np.ascontiguousarray(idx, np.int64)
    dist = _f32m(dist)
    out = np.empty(idx.shape[0], np.float32)
    load().orc_local_radii(_p(idx), _p(dist), idx.shape[0], idx.shape[1], var_shift, _p(out))
    return out


def transform(train, train_emb, q, a: float, b: float, **kw):
    train, q = _f32m(train), _f32m(q)
    train_emb = _f32m(train_emb)
    p = _params(**kw)
    out = np.empty((q.shape[0], p.n_components), np.float32)
    load().orc_transform(_p(train), train.shape[0], _p(train_emb), _p(q), q.shape[0],
                         q.shape[1], ctypes.byref(p), a, b, _p(out))
    return out


def transform_graph(train, train_emb, q, **kw):
    """sigma, rho, pruned bipartite edges (head, tail, weight) and the
    initial positions of transform_from_knn before its SGD."""
    train, q = _f32m(train), _f32m(q)
    train_emb = _f32m(train_emb)
    p = _params(**kw)
    nq = q.shape[0]
    cap = nq * max(1, p.n_neighbors)
    sig = np.empty(nq, np.float32)
    rho = np.empty(nq, np.float32)
    h = np.empty(cap, np.int32)
    t = np.empty(cap, np.int32)
    w = np.empty(cap, np.float32)
    init = np.empty((nq, p.n_components), np.float32)
    m = load().orc_transform_graph(_p(train), train.shape[0], _p(train_emb), _p(q), nq,
                                   q.shape[1], ctypes.byref(p), _p(sig), _p(rho), _p(h), _p(t),
                                   _p(w), cap, _p(init))
    if m < 0:
        raise ValueError("edge capacity too small")
    return sig, rho, h[:m].copy(), t[:m].copy(), w[:m].copy(), init


def optimize_layout_transform(emb, base, heads, tails, weights, n_epochs, a, b, alpha, neg_rate,
                              repulsion, seed):
    emb = np.array(emb, dtype=np.float32, copy=True, order="C")
    base = _f32m(base)
    heads = np.ascontiguousarray(heads, np.int32)
    tails = np.ascontiguousarray(tails, np.int32)
    weights = _f32m(weights)
    load().orc_optimize_layout_transform(_p(emb), emb.shape[0], emb.shape[1], _p(base),
                                         base.shape[0], _p(heads), _p(tails), _p(weights),
                                         heads.shape[0], n_epochs, a, b, alpha, neg_rate,
                                         repulsion, seed)
    return emb


def laplacians(n, heads, tails, weights):
    heads = np.ascontiguousarray(heads, np.int32)
    tails = np.ascontiguousarray(tails, np.int32)
    weights = _f32m(weights)
    l1 = np.empty((n, n), np.float64)
    l2 = np.empty((n, n), np.float64)
    st = load().orc_laplacians(n, _p(heads), _p(tails), _p(weights), heads.shape[0], _p(l1),
                               _p(l2))
    if st != 0:
        raise ValueError("empty graph")
    return l1, l2


def rng_u64(seed: int, count: int):
    out = np.empty(count, np.uint64)
    load().orc_rng_u64(seed, count, _p(out))
    return out
