"""tups_b200: the TUPS parquet-loop hot path on one NVIDIA B200 (sm_100a).

All compute runs in ``libtups_b200.so`` (hand-written CUDA, C ABI in
``include/tups_b200.h``); this package is the host-side mirror of the
reference's Fortran module entry points.
"""
from ._lib import TupsError, exported_symbols, load
from .parquet import CHANNELS, Params, Solver, read_prms

__all__ = ["TupsError", "Params", "Solver", "read_prms", "load", "exported_symbols", "CHANNELS"]
