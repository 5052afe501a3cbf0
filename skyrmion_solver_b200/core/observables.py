"""Host observable routines with the reference's signatures
(e.g. skyrmion_solver ``th/nuclear_skyrme/observables.py:26-50, 408-474``).

``compute_energy`` / ``compute_skyrmion_number`` evaluate the per-site density
and its compensated FP64 sum in one fused launch.  Like the reference they
leave ``en`` and ``entmp`` zeroed on return.
"""
from __future__ import annotations

import ctypes

from .. import _lib
from .._lib import dptr, f64p, host_params, i32p, stream_ptr
from .utils import pick_scratch, _numel


def _zero(*bufs):
    for b in bufs:
        if b is None:
            continue
        z = getattr(b, "zero_", None)
        if z is not None:
            z()
        else:  # __cuda_array_interface__ arrays (e.g. Numba)
            b[:] = 0.0


def _total(fn, theory_id, Field, en, entmp, gridsum_partial, p_i, p_f):
    hi, hf = host_params(p_i, p_f)
    scratch = pick_scratch(gridsum_partial)
    out = ctypes.c_double(0.0)
    _lib.call(fn, theory_id, i32p(hi), len(hi), f64p(hf), len(hf), dptr(Field), dptr(scratch), _numel(scratch),
              ctypes.byref(out), stream_ptr())
    _zero(en, entmp)
    return float(out.value)


class EnergyObservable:
    """compute_energy(Field, d1fd1x, en, entmp, gridsum_partial, p_i_d, p_f_d, p_i_h, p_f_h) -> float"""

    def __init__(self, theory_id):
        self.theory_id = theory_id

    def __call__(self, Field, d1fd1x, en, entmp, gridsum_partial, p_i_d, p_f_d, p_i_h=None, p_f_h=None):
        p_i = p_i_h if p_i_h is not None else p_i_d
        p_f = p_f_h if p_f_h is not None else p_f_d
        return _total("sky_total_energy", self.theory_id, Field, en, entmp, gridsum_partial, p_i, p_f)


class BaryonObservable:
    """compute_skyrmion_number(Field, d1fd1x, en, entmp, gridsum_partial, p_i_d, p_f_d, p_i_h) -> float"""

    def __init__(self, theory_id):
        self.theory_id = theory_id

    def __call__(self, Field, d1fd1x, en, entmp, gridsum_partial, p_i_d, p_f_d, p_i_h=None, p_f_h=None):
        p_i = p_i_h if p_i_h is not None else p_i_d
        p_f = p_f_h if p_f_h is not None else p_f_d
        return _total("sky_total_baryon", self.theory_id, Field, en, entmp, gridsum_partial, p_i, p_f)
