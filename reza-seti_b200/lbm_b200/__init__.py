"""B200 lattice-Boltzmann engine: Python binding of the C ABI (include/lbm_b200.h)."""
from .capi import LbmError, lib  # noqa: F401
from .engine import Engine, Simulation  # noqa: F401
