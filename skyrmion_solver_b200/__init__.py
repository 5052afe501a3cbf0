"""skyrmion_solver_b200 — B200-native (sm_100a) lattice engine for skyrmion_solver's hot path.

The reference's theory-module API is mirrored (``theories.load_theory``,
``core.simulation.Simulation``, per-theory ``params`` / ``kernels`` /
``observables`` / ``initial_config``); compute runs in hand-written CUDA
kernels behind the C ABI ``include/skyrmion_b200.h`` (``libskyrmion_b200.so``).
"""
from __future__ import annotations

__version__ = "0.1.0"


def library():
    """Load the native library (raises if it is missing: there is no fallback)."""
    from . import _lib
    return _lib.load()
