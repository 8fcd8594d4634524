"""Drop-in module name of the estimator layer (``umapers._api``)."""
from umapers_b200._api import *  # noqa: F401,F403
from umapers_b200._api import _PARAM_NAMES, UmapCore  # noqa: F401
