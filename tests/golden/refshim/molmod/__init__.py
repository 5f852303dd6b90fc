"""Shim: molmod names used by the reference, backed by cmmdft_b200.units."""
from . import units, constants  # noqa: F401
