"""Drop-in import name: ``import umapers`` resolves to the B200 engine."""
from umapers_b200 import AlignedUmap, ParametricUmap, Umap, UmapKwargs, __version__, fit_transform

__all__ = ["Umap", "ParametricUmap", "AlignedUmap", "UmapKwargs", "fit_transform", "__version__"]
