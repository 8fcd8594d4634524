"""Drop-in module name of the estimator layer (``umapers._api``).

The name refers to the engine's own facade module object, so attributes set
on ``umapers._api`` (for example a patched ``UmapCore``) are the ones
``Umap`` uses.
"""
import sys

from umapers_b200 import _api as _facade

sys.modules[__name__] = _facade
