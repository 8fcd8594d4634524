"""Drop-in module name of the diagnostics helpers (``umapers.diagnostics``)."""
from umapers_b200.diagnostics import knn_preservation, quality, trustworthiness_report  # noqa: F401
