"""umapers_b200: a single-GPU UMAP engine for NVIDIA B200 with the umapers API.

``Umap`` / ``fit_transform`` keep the surface of the reference package
``umapers``; every compute stage runs in libumapb200.so (hand-written
sm_100a kernels behind a C ABI, include/umapb200.h).
"""
from ._api import AlignedUmap, ParametricUmap, Umap, UmapKwargs, fit_transform
from ._umapers import __version__

__all__ = ["Umap", "ParametricUmap", "AlignedUmap", "UmapKwargs", "fit_transform", "__version__"]
