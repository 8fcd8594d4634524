"""Small, self-contained GPU cases for profiling one kernel family at a time.

    python -m umapers_b200.profiling knn_tc [--rows 262144] [--dim 64]
    python -m umapers_b200.profiling surrogate [--rows 262144] [--fit-rows 50000]
    python -m umapers_b200.profiling fit [--rows 262144] [--dim 64]
    python -m umapers_b200.profiling sparse [--rows 200000] [--dim 2000]

Each case runs once untimed, then once inside an NVTX range named after the
case, so a profiler can be limited to the measured launches, e.g.

    ncu --clock-control none --nvtx --nvtx-include "knn_tc/" \
        -k regex:tc_knn_kernel -c 1 ...

and prints the wall time of the measured run.  Inputs are the seeded
synthetic mixtures of ``umapers_b200.workloads``; the cases are sized to stay
far below device memory (a few GB at most) while their operands exceed L2.
"""
from __future__ import annotations

import argparse
import ctypes
import time

import numpy as np

from . import _lib, workloads


class _Range:
    """NVTX push/pop around a synchronised, wall-timed region."""

    def __init__(self, name: str):
        self.name = name
        self.dt = 0.0

    def __enter__(self):
        import torch

        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push(self.name)
        self.t0 = time.perf_counter()
        return self

    def __exit__(self, *exc):
        import torch

        torch.cuda.synchronize()
        self.dt = time.perf_counter() - self.t0
        torch.cuda.nvtx.range_pop()


def case_knn_tc(rows: int, dim: int) -> None:
    """Exact kNN (k = 15) of `rows` anisotropic-mixture rows on the tensor path."""
    x = workloads.anisotropic_mixture(rows, dim, 50, seed=11)
    lib = _lib.load()
    idx = np.empty((rows, 15), np.int64)
    dist = np.empty((rows, 15), np.float32)
    fb = ctypes.c_int64(0)

    def run():
        _lib.check(lib.umapb_knn_exact(x.ctypes.data, rows, dim, 15, 0, 1, idx.ctypes.data,
                                       dist.ctypes.data, ctypes.byref(fb)))

    run()
    with _Range("knn_tc") as r:
        run()
    print(f"knn_tc rows={rows} dim={dim}: {r.dt:.4f} s, fallback rows {fb.value}")


def case_surrogate(rows: int, fit_rows: int = 50_000) -> None:
    """Surrogate transform of `rows` queries (128 features), gated rows
    recomputed by the plain transform, after training on a `fit_rows`-row fit
    of the same mixture."""
    import torch

    from umapers import Umap

    fit, query = workloads.transform_mixture(n_fit=fit_rows, n_query=rows, d=128)
    m = Umap(n_neighbors=15, random_seed=5, ann_mode="exact")
    m.fit(fit)
    m.fit_surrogate(batch_size=1024)
    lib = _lib.load()
    q = torch.from_numpy(query).cuda()
    out = torch.empty((rows, 2), dtype=torch.float32, device="cuda")
    nf = ctypes.c_int64(0)

    def run():
        _lib.check(lib.umapb_surrogate_transform_device(m._core._handle, q.data_ptr(), rows, 128,
                                                        1, out.data_ptr(), None,
                                                        ctypes.byref(nf)))

    run()
    with _Range("surrogate") as r:
        run()
    print(f"surrogate transform rows={rows}: {r.dt:.4f} s, gated rows {nf.value}")


def case_sparse(rows: int, dim: int) -> None:
    """Exact cosine kNN (k = 30) of `rows` CSR rows with about 20 LogNormal
    values each among `dim` columns."""
    x = workloads.sparse_lognormal_csr(rows, dim, 20, seed=3)
    lib = _lib.load()
    ip = np.ascontiguousarray(x.indptr, np.int64)
    ix = np.ascontiguousarray(x.indices, np.int64)
    dv = np.ascontiguousarray(x.data, np.float32)
    idx = np.empty((rows, 30), np.int64)
    dist = np.empty((rows, 30), np.float32)

    def run():
        _lib.check(lib.umapb_knn_csr(ip.ctypes.data, ix.ctypes.data, dv.ctypes.data, rows, dim,
                                     30, 2, idx.ctypes.data, dist.ctypes.data))

    run()
    with _Range("sparse") as r:
        run()
    print(f"sparse kNN rows={rows} dim={dim} nnz={x.nnz}: {r.dt:.4f} s")


def case_fit(rows: int, dim: int) -> None:
    """One complete fit (exact kNN, spectral init, 200 epochs)."""
    from umapers import Umap

    x = workloads.anisotropic_mixture(rows, dim, 50, seed=11)
    m = Umap(n_neighbors=15, n_epochs=200, ann_mode="exact")
    m.fit(x)
    with _Range("fit") as r:
        m.fit(x)
    print(f"fit rows={rows} dim={dim}: {r.dt:.4f} s")


def main() -> None:
    ap = argparse.ArgumentParser(description="profiling cases of libumapb200")
    ap.add_argument("case", choices=["knn_tc", "surrogate", "fit", "sparse"])
    ap.add_argument("--rows", type=int, default=262_144)
    ap.add_argument("--dim", type=int, default=None)
    ap.add_argument("--fit-rows", type=int, default=50_000, help="surrogate case: fitted rows")
    a = ap.parse_args()
    if a.dim is None:
        a.dim = 2000 if a.case == "sparse" else 64
    if a.case == "knn_tc":
        case_knn_tc(a.rows, a.dim)
    elif a.case == "surrogate":
        case_surrogate(a.rows, a.fit_rows)
    elif a.case == "sparse":
        case_sparse(a.rows, a.dim)
    else:
        case_fit(a.rows, a.dim)


if __name__ == "__main__":
    main()
