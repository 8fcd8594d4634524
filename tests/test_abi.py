"""libumapb200.so loads without a GPU and exports every entry point that
include/umapb200.h declares; host-only entry points run here."""
import ctypes
import re
from pathlib import Path

import numpy as np

from umapers_b200 import _lib

ROOT = Path(__file__).resolve().parents[1]


def _declared() -> set[str]:
    text = (ROOT / "include/umapb200.h").read_text()
    return set(re.findall(r"^(?:const char\*|int32_t|int64_t|uint64_t|void)\s+(umapb_\w+)\(", text, re.M))


def test_header_declares_the_bound_entry_points():
    assert _declared() == set(_lib.SIGNATURES), _declared() ^ set(_lib.SIGNATURES)


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    for name in _declared():
        assert hasattr(lib, name), name


def test_version_and_defaults():
    lib = _lib.load()
    assert lib.umapb_abi_version() == 2
    assert lib.umapb_version().decode().startswith("1.1.4")
    p = _lib.Params()
    lib.umapb_params_default(ctypes.byref(p))
    # UmapParams::default (rust_umap/src/lib.rs:170-195)
    assert (p.n_neighbors, p.n_components, p.n_epochs) == (15, 2, -1)
    assert (p.learning_rate, p.set_op_mix_ratio, p.repulsion_strength) == (1.0, 1.0, 1.0)
    assert np.float32(p.min_dist) == np.float32(0.1) and p.spread == 1.0
    assert (p.negative_sample_rate, p.random_seed, p.init) == (5, 42, 1)
    assert (p.use_approximate_knn, p.approx_knn_candidates, p.approx_knn_iters,
            p.approx_knn_threshold) == (1, 50, 14, 4096)
    assert np.float32(p.dens_lambda) == 2.0 and np.float32(p.dens_frac) == np.float32(0.3)


def test_find_ab_params_through_the_abi_matches_reference_bits(pins):
    lib = _lib.load()
    for case in pins["find_ab_params"]:
        a, b = ctypes.c_float(), ctypes.c_float()
        assert lib.umapb_find_ab_params(case["spread"], case["min_dist"], ctypes.byref(a),
                                        ctypes.byref(b)) == 0
        assert int(np.float32(a.value).view(np.uint32)) == case["a_bits"]
        assert int(np.float32(b.value).view(np.uint32)) == case["b_bits"]


def test_create_destroy_needs_no_device():
    lib = _lib.load()
    p = _lib.Params()
    lib.umapb_params_default(ctypes.byref(p))
    h = ctypes.c_void_p()
    assert lib.umapb_create(ctypes.byref(p), ctypes.byref(h)) == 0
    assert lib.umapb_n_features(h) == -1 and lib.umapb_n_components(h) == 2
    lib.umapb_destroy(h)


def test_ann_switch_matches_reference_pins(pins):
    # auto_approximate_knn_delays_crossover_beyond_public_threshold
    # (rust_umap/src/lib.rs:5814-5840): default parameters, threshold 4096
    lib = _lib.load()
    p = _lib.Params()
    lib.umapb_params_default(ctypes.byref(p))
    assert len(pins["ann_switch"]) == 5
    for case in pins["ann_switch"]:
        got = lib.umapb_should_use_approximate_knn(ctypes.byref(p), case["n"], case["d"])
        assert bool(got) == case["expect"], case
    # the switch is off entirely without use_approximate_knn, and any size
    # above a zero threshold takes the approximate path
    p.use_approximate_knn = 0
    assert lib.umapb_should_use_approximate_knn(ctypes.byref(p), 10 ** 6, 64) == 0
    p.use_approximate_knn = 1
    p.approx_knn_threshold = 0
    assert lib.umapb_should_use_approximate_knn(ctypes.byref(p), 2, 64) == 1
