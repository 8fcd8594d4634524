"""Drop-in module name of the engine class (``umapers._umapers.UmapCore``)."""
from umapers_b200._umapers import AlignedUmapCore, ParametricUmapCore, UmapCore, __version__

__all__ = ["UmapCore", "ParametricUmapCore", "AlignedUmapCore", "__version__"]
