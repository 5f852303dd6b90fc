"""Shim: the reference imports matplotlib at module level only for plots."""
from . import cm, pyplot  # noqa: F401
__version__ = "0.0-shim"
