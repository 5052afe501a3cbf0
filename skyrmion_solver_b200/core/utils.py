"""Launch helpers and reductions with the reference's interface
(skyrmion_solver ``core/utils.py:176-424``).

The reductions are deterministic FP64 (compensated sum, signed max, min) and run
as a single sm_100a launch each; the reference's block-partial buffers are
accepted and used as scratch when large enough.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .. import _lib
from .._lib import dptr, stream_ptr
from .launch import SetFieldZeroKernel

MAX_TPB = 1024

set_field_zero_kernel = SetFieldZeroKernel()

_scratch_cache = {}


def scratch_doubles() -> int:
    return int(_lib.load().sky_reduce_scratch_size(0))


def reduction_scratch(device=None, slots: int = 1):
    """A cached per-device scratch buffer for the library's reductions."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
    key = (dev.index, slots)
    buf = _scratch_cache.get(key)
    if buf is None:
        buf = torch.zeros(slots * scratch_doubles(), dtype=torch.float64, device=dev)
        _scratch_cache[key] = buf
    return buf


def _numel(buf) -> int:
    n = getattr(buf, "numel", None)
    if callable(n):
        return int(n())
    cai = buf.__cuda_array_interface__
    return int(np.prod(cai["shape"]))


def pick_scratch(partial, slots: int = 1):
    """Use the caller's partial buffer when it is a float64 buffer large enough, else the cache."""
    need = slots * scratch_doubles()
    if partial is not None:
        try:
            if _numel(partial) >= need:
                return partial
        except (AttributeError, TypeError):
            pass
    return reduction_scratch(slots=slots)


def launch_3d(p_i_h, threads=(8, 8, 8)):
    """Grid covering the lattice (core/utils.py:176-199); kept for API compatibility."""
    xlen, ylen, zlen = int(p_i_h[0]), int(p_i_h[1]), int(p_i_h[2])
    bx, by, bz = threads
    grid = ((xlen + bx - 1) // bx, (ylen + by - 1) // by, (zlen + bz - 1) // bz)
    return grid, (bx, by, bz)


def _reduce(fn, var_d, partial_d, size):
    scratch = pick_scratch(partial_d)
    out = ctypes.c_double(0.0)
    _lib.call(fn, dptr(var_d), int(size), dptr(scratch), _numel(scratch), ctypes.byref(out), None, stream_ptr())
    return float(out.value)


def compute_sum(var_d, partial_d, size: int) -> float:
    """Sum of the first ``size`` entries (core/utils.py:321-346)."""
    return _reduce("sky_sum", var_d, partial_d, size)


def compute_max(var_d, partial_d, size: int) -> float:
    """Signed maximum of the first ``size`` entries (core/utils.py:348-373)."""
    return _reduce("sky_max", var_d, partial_d, size)


def compute_min(var_d, partial_d, size: int) -> float:
    """Minimum of the first ``size`` entries (core/utils.py:375-400)."""
    return _reduce("sky_min", var_d, partial_d, size)


def compute_max_field(EnergyGradient, max_partial, p_i_h) -> float:
    """Signed maximum over the flattened field (core/utils.py:402-424)."""
    return _reduce("sky_max", EnergyGradient, max_partial, int(p_i_h[7]))
