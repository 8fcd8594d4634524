"""ctypes bindings of libumapb200.so (declared in include/umapb200.h).

The shared library is built in-tree by ``python -m umapers_b200.build`` (or
``__graft_entry__.build()``).  Loading fails loudly when it is missing: there
is no CPU fallback behind this package.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

_PKG = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("UMAPB200_LIB", _PKG / "libumapb200.so"))

# umapb_status (include/umapb200.h)
OK = 0
ERR_EMPTY_DATA = 1
ERR_NEED_TWO_SAMPLES = 2
ERR_INCONSISTENT_DIMS = 3
ERR_FEATURE_MISMATCH = 4
ERR_EMBEDDING_DIM_MISMATCH = 5
ERR_NOT_FITTED = 6
ERR_INVALID_PARAMETER = 7
ERR_CUDA = 8
ERR_OUT_OF_MEMORY = 9

METRICS = {
    "euclidean": 0,
    "manhattan": 1,
    "cosine": 2,
    "chebyshev": 3,
    "minkowski": 4,
    "correlation": 5,
    "canberra": 6,
    "braycurtis": 7,
}
KNN_BACKENDS = {"auto": 0, "tensor": 1, "plain": 2}


class Params(ctypes.Structure):
    """umapb_params."""

    _fields_ = [
        ("n_neighbors", ctypes.c_int64),
        ("n_components", ctypes.c_int64),
        ("n_epochs", ctypes.c_int64),
        ("metric", ctypes.c_int32),
        ("metric_p", ctypes.c_float),
        ("learning_rate", ctypes.c_float),
        ("min_dist", ctypes.c_float),
        ("spread", ctypes.c_float),
        ("local_connectivity", ctypes.c_float),
        ("set_op_mix_ratio", ctypes.c_float),
        ("repulsion_strength", ctypes.c_float),
        ("negative_sample_rate", ctypes.c_int64),
        ("random_seed", ctypes.c_uint64),
        ("init", ctypes.c_int32),
        ("use_approximate_knn", ctypes.c_int32),
        ("approx_knn_candidates", ctypes.c_int64),
        ("approx_knn_iters", ctypes.c_int64),
        ("approx_knn_threshold", ctypes.c_int64),
        ("densmap", ctypes.c_int32),
        ("dens_lambda", ctypes.c_float),
        ("dens_frac", ctypes.c_float),
        ("dens_var_shift", ctypes.c_float),
        ("output_dens", ctypes.c_int32),
        ("knn_backend", ctypes.c_int32),
    ]


TIMING_FIELDS = (
    "validation_sec",
    "knn_sec",
    "curve_params_sec",
    "knn_validate_trim_sec",
    "smooth_knn_sec",
    "density_original_sec",
    "membership_sec",
    "symmetrize_sec",
    "target_intersection_sec",
    "prune_sec",
    "init_sec",
    "optimize_sec",
    "density_embedding_sec",
    "output_copy_sec",
    "store_state_sec",
    "total_sec",
)


class Timings(ctypes.Structure):
    """umapb_timings (the FitTimingBreakdown fields)."""

    _fields_ = [(name, ctypes.c_double) for name in TIMING_FIELDS]


class FitInfo(ctypes.Structure):
    """umapb_fit_info."""

    _fields_ = [
        ("used_approximate_knn", ctypes.c_int32),
        ("knn_backend_used", ctypes.c_int32),
        ("n_samples", ctypes.c_int64),
        ("n_features", ctypes.c_int64),
        ("n_epochs", ctypes.c_int64),
        ("n_edges", ctypes.c_int64),
        ("knn_fallback_rows", ctypes.c_int64),
        ("n_components_graph", ctypes.c_int64),
        ("knn_kernel_sec", ctypes.c_double),
        ("sgd_edge_samples", ctypes.c_double),
        ("knn_second_pass_rows", ctypes.c_int64),
        ("stage_wait_sec", ctypes.c_double),
        ("stage_host_sec", ctypes.c_double),
        ("sgd_kernel_sec", ctypes.c_double),
    ]


class SurrogateParams(ctypes.Structure):
    """umapb_surrogate_params."""

    _fields_ = [
        ("hidden", ctypes.c_int64),
        ("epochs", ctypes.c_int64),
        ("batch_size", ctypes.c_int64),
        ("learning_rate", ctypes.c_float),
        ("mse_weight", ctypes.c_float),
        ("edge_loss_weight", ctypes.c_float),
        ("negatives", ctypes.c_int64),
        ("holdout_fraction", ctypes.c_float),
        ("n_anchors", ctypes.c_int64),
        ("fallback_radius", ctypes.c_float),
        ("max_cell_failure", ctypes.c_float),
        ("seed", ctypes.c_uint64),
    ]


SURROGATE_INFO_FIELDS = (
    ("n_train", ctypes.c_int64),
    ("n_holdout", ctypes.c_int64),
    ("steps", ctypes.c_int64),
    ("n_anchors", ctypes.c_int64),
    ("cells_trusted", ctypes.c_int64),
    ("radius", ctypes.c_double),
    ("train_sec", ctypes.c_double),
    ("calibrate_sec", ctypes.c_double),
    ("first_epoch_loss", ctypes.c_double),
    ("final_epoch_loss", ctypes.c_double),
    ("holdout_rmse", ctypes.c_double),
    ("holdout_median_error", ctypes.c_double),
    ("holdout_within_radius", ctypes.c_double),
    ("holdout_gated", ctypes.c_double),
)


class SurrogateInfo(ctypes.Structure):
    """umapb_surrogate_info."""

    _fields_ = list(SURROGATE_INFO_FIELDS)


class MlpBatch(ctypes.Structure):
    """umapb_mlp_batch."""

    _fields_ = [
        ("batch", ctypes.c_int64),
        ("n_features", ctypes.c_int64),
        ("hidden", ctypes.c_int64),
        ("n_out", ctypes.c_int64),
        ("x", ctypes.c_void_p),
        ("targets", ctypes.c_void_p),
        ("params", ctypes.c_void_p),
        ("teacher", ctypes.c_void_p),
        ("n_teacher", ctypes.c_int64),
        ("edge_ptr", ctypes.c_void_p),
        ("edge_tail", ctypes.c_void_p),
        ("edge_weight", ctypes.c_void_p),
        ("neg_tail", ctypes.c_void_p),
        ("n_neg", ctypes.c_int64),
        ("a", ctypes.c_float),
        ("b", ctypes.c_float),
        ("mse_weight", ctypes.c_float),
        ("edge_loss_weight", ctypes.c_float),
        ("neg_scale", ctypes.c_float),
        ("out_shift", ctypes.c_void_p),
        ("out_scale", ctypes.c_void_p),
    ]


_f32p = ctypes.POINTER(ctypes.c_float)
_i64p = ctypes.POINTER(ctypes.c_int64)
_i32p = ctypes.POINTER(ctypes.c_int32)
_vp = ctypes.c_void_p
_i64 = ctypes.c_int64
_i32 = ctypes.c_int32
_f32 = ctypes.c_float
_u64 = ctypes.c_uint64

# name -> (restype, argtypes); the full list of entry points of the header.
SIGNATURES = {
    "umapb_version": (ctypes.c_char_p, []),
    "umapb_abi_version": (_i32, []),
    "umapb_should_use_approximate_knn": (_i32, [_vp, _i64, _i64]),
    "umapb_last_error": (ctypes.c_char_p, []),
    "umapb_kernel_launches": (_u64, []),
    "umapb_pool_bytes": (_i32, [_vp, _vp]),
    "umapb_params_default": (None, [ctypes.POINTER(Params)]),
    "umapb_create": (_i32, [ctypes.POINTER(Params), ctypes.POINTER(_vp)]),
    "umapb_destroy": (None, [_vp]),
    "umapb_fit": (_i32, [_vp, _vp, _i64, _i64]),
    "umapb_fit_transform": (_i32, [_vp, _vp, _i64, _i64, _vp]),
    "umapb_fit_supervised": (_i32, [_vp, _vp, _i64, _i64, _vp, _i64, _f32, _i64]),
    "umapb_inverse_transform": (_i32, [_vp, _vp, _i64, _i64, _vp]),
    "umapb_fit_transform_supervised": (_i32, [_vp, _vp, _i64, _i64, _vp, _i64, _f32, _i64, _vp]),
    "umapb_fit_transform_stateless": (_i32, [ctypes.POINTER(Params), _vp, _i64, _i64, _vp]),
    "umapb_fit_transform_with_knn": (
        _i32,
        [_vp, _vp, _i64, _i64, _vp, _i64, _i64, _vp, _i64, _i64, _i32, _i32, _vp],
    ),
    "umapb_transform": (_i32, [_vp, _vp, _i64, _i64, _vp]),
    "umapb_transform_graph": (_i32, [_vp, _vp, _i64, _i64, _vp, _vp, _vp, _vp, _vp, _i64, _vp,
                                     _vp]),
    "umapb_fit_csr": (_i32, [_vp, _vp, _vp, _vp, _i64, _i64]),
    "umapb_fit_transform_csr": (_i32, [_vp, _vp, _vp, _vp, _i64, _i64, _vp]),
    "umapb_fit_transform_csr_stateless": (_i32, [_vp, _vp, _vp, _vp, _i64, _i64, _vp]),
    "umapb_transform_csr": (_i32, [_vp, _vp, _vp, _vp, _i64, _i64, _vp]),
    "umapb_knn_csr": (_i32, [_vp, _vp, _vp, _i64, _i64, _i64, _i32, _vp, _vp]),
    "umapb_knn_csr_query": (
        _i32, [_vp, _vp, _vp, _i64, _vp, _vp, _vp, _i64, _i64, _i64, _i32, _vp, _vp]),
    "umapb_profile_fit_transform": (
        _i32,
        [_vp, _vp, _i64, _i64, _vp, ctypes.POINTER(Timings), ctypes.POINTER(FitInfo)],
    ),
    "umapb_fit_transform_device": (
        _i32,
        [_vp, _vp, _i64, _i64, _vp, ctypes.POINTER(Timings), ctypes.POINTER(FitInfo)],
    ),
    "umapb_transform_device": (_i32, [_vp, _vp, _i64, _i64, _vp]),
    "umapb_n_components": (_i64, [_vp]),
    "umapb_n_neighbors": (_i64, [_vp]),
    "umapb_n_features": (_i64, [_vp]),
    "umapb_n_samples": (_i64, [_vp]),
    "umapb_get_embedding": (_i32, [_vp, _vp, _i64, _i64]),
    "umapb_get_ab": (_i32, [_vp, _f32p, _f32p]),
    "umapb_has_radii": (_i32, [_vp]),
    "umapb_get_radii": (_i32, [_vp, _vp, _vp, _i64]),
    "umapb_find_ab_params": (_i32, [_f32, _f32, _f32p, _f32p]),
    "umapb_knn_exact": (_i32, [_vp, _i64, _i64, _i64, _i32, _i32, _vp, _vp, _i64p]),
    "umapb_knn_exact_noalloc": (_i32, [_vp, _i64, _i64, _i64, _vp, _vp, _vp]),
    "umapb_knn_query": (_i32, [_vp, _i64, _vp, _i64, _i64, _i64, _i32, _i32, _vp, _vp]),
    "umapb_nndescent": (_i32, [_vp, _i64, _i64, _i64, _i32, _i64, _i64, _u64, _vp, _vp, _i64p,
                               _i64p, ctypes.POINTER(ctypes.c_double)]),
    "umapb_nndescent_csr": (_i32, [_vp, _vp, _vp, _i64, _i64, _i64, _i32, _i64, _i64, _u64, _vp,
                                   _vp, _i64p, _i64p, ctypes.POINTER(ctypes.c_double)]),
    "umapb_smooth_knn_dist": (_i32, [_vp, _i64, _i64, _f32, _f32, _f32, _i32, _vp, _vp]),
    "umapb_fuzzy_graph": (
        _i32,
        [_vp, _vp, _i64, _i64, _f32, _f32, _i64, _vp, _vp, _vp, _i64, _i64p, _vp, _vp],
    ),
    "umapb_fuzzy_graph_supervised": (
        _i32,
        [_vp, _vp, _i64, _i64, _f32, _f32, _i64, _vp, _f32, _vp, _vp, _vp, _i64, _i64p],
    ),
    "umapb_spectral_init": (
        _i32,
        [_vp, _i64, _i64, _vp, _vp, _vp, _i64, _i64, _u64, _vp, _i32p],
    ),
    "umapb_optimize_layout": (
        _i32,
        [_vp, _i64, _i64, _vp, _vp, _vp, _i64, _i64, _f32, _f32, _f32, _i64, _f32, _u64],
    ),
    "umapb_surrogate_params_default": (None, [ctypes.POINTER(SurrogateParams)]),
    "umapb_surrogate_fit": (
        _i32,
        [_vp, ctypes.POINTER(SurrogateParams), ctypes.POINTER(SurrogateInfo)],
    ),
    "umapb_surrogate_ready": (_i32, [_vp]),
    "umapb_surrogate_transform": (_i32, [_vp, _vp, _i64, _i64, _i32, _vp, _vp, _i64p]),
    "umapb_surrogate_transform_device": (_i32, [_vp, _vp, _i64, _i64, _i32, _vp, _vp, _i64p]),
    "umapb_surrogate_loss_history": (_i32, [_vp, _vp, _i64, _i64p]),
    "umapb_mlp_grad": (_i32, [ctypes.POINTER(MlpBatch), _vp, _vp, _vp]),
}

_LIB: ctypes.CDLL | None = None


class UmapbError(Exception):
    """Base class for errors raised by the engine."""


def load() -> ctypes.CDLL:
    """Load libumapb200.so once and declare every entry point."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not LIB_PATH.exists():
        raise ImportError(
            f"{LIB_PATH} is missing: build the CUDA engine with `python -m umapers_b200.build`"
        )
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (restype, argtypes) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = restype
        fn.argtypes = argtypes
    _LIB = lib
    return lib


def last_error() -> str:
    msg = load().umapb_last_error()
    return msg.decode() if msg else ""


def check(status: int) -> None:
    """Raise the exception the reference binding maps a status to
    (umap_rs/src/lib.rs:147-157): RuntimeError for NotFitted and device
    failures, ValueError for everything else."""
    if status == OK:
        return
    msg = last_error() or f"umapb status {status}"
    if status in (ERR_NOT_FITTED, ERR_CUDA):
        raise RuntimeError(msg)
    if status == ERR_OUT_OF_MEMORY:
        raise MemoryError(msg)
    raise ValueError(msg)


def ptr(arr) -> int:
    """Address of a NumPy array's data (None -> NULL)."""
    if arr is None:
        return None
    return arr.ctypes.data
