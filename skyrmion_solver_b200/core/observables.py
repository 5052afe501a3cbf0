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


def _moments(theory_id, Field, gridsum_partial, p_i, p_f):
    import numpy as np
    hi, hf = host_params(p_i, p_f)
    scratch = pick_scratch(gridsum_partial)
    out = np.zeros(9)
    _lib.call("sky_baryon_moments", theory_id, i32p(hi), len(hi), f64p(hf), len(hf), dptr(Field), dptr(scratch),
              _numel(scratch), f64p(out), stream_ptr())
    return out


class CenterOfMassObservable:
    """compute_center_of_mass(Field, grid, d1fd1x, obs4, tensor_scratch, entmp, gridsum_partial, p_i_d, p_f_d,
    p_i_h) -> ndarray (3,): sum b r / sum b over the baryon density b (grid r = h * index), zeros when
    |sum b| < 1e-30 (th/nuclear_skyrme/observables.py:182-221).  One fused device pass
    (sky_baryon_moments); obs4 and tensor_scratch are not needed and left untouched."""

    def __init__(self, theory_id):
        self.theory_id = theory_id

    def __call__(self, Field, grid, d1fd1x, obs4, tensor_scratch, entmp, gridsum_partial, p_i_d, p_f_d, p_i_h=None):
        import numpy as np
        m = _moments(self.theory_id, Field, gridsum_partial, p_i_h if p_i_h is not None else p_i_d, p_f_d)
        if abs(m[0]) < 1.0e-30:
            return np.zeros(3, dtype=np.float64)
        return m[1:4] / m[0]


class RmsRadiusObservable:
    """compute_rms_radius(Field, grid, d1fd1x, en, entmp, gridsum_partial, obs4, tensor_scratch, com_d, p_i_d,
    p_f_d, p_i_h) -> float: sqrt(max(sum |b| |r - COM|^2 / sum b, 0)), with the centre of mass also
    written to com_d (th/nuclear_skyrme/observables.py:224-270).  One fused device pass; en and entmp
    are left zeroed, as the reference's energy / baryon sums leave them."""

    def __init__(self, theory_id):
        self.theory_id = theory_id

    def __call__(self, Field, grid, d1fd1x, en, entmp, gridsum_partial, obs4, tensor_scratch, com_d, p_i_d, p_f_d,
                 p_i_h=None):
        import math
        import numpy as np
        m = _moments(self.theory_id, Field, gridsum_partial, p_i_h if p_i_h is not None else p_i_d, p_f_d)
        B = m[0]
        com = np.zeros(3) if abs(B) < 1.0e-30 else m[1:4] / B
        if com_d is not None:
            import torch
            if isinstance(com_d, torch.Tensor):
                com_d.copy_(torch.from_numpy(com))
            else:
                com_d.copy_to_device(com)
        _zero(en, entmp)
        if abs(B) < 1.0e-30:
            return 0.0
        num = m[8] - 2.0 * float(np.dot(com, m[5:8])) + float(np.dot(com, com)) * m[4]
        return math.sqrt(max(num / B, 0.0))


# ---------------------------------------------------------------------------
# nuclear-model inertia and shape diagnostics (th/nuclear_skyrme/observables.py:273-487)
# ---------------------------------------------------------------------------
def _sym(v6):
    import numpy as np
    a, b, c, d, e, f = v6
    return np.array([[a, b, c], [b, d, e], [c, e, f]], dtype=np.float64)


def _nuclear_diag(theory_id, Field, gridsum_partial, p_i, p_f, moments=None):
    """(centre of mass, the 28 fused sums of sky_nuclear_diagnostics).  `moments`: the nine
    baryon moments of the same field when the caller already has them (sky_baryon_moments)."""
    import numpy as np
    m = _moments(theory_id, Field, gridsum_partial, p_i, p_f) if moments is None else moments
    com = np.zeros(3) if abs(m[0]) < 1.0e-30 else m[1:4] / m[0]
    hi, hf = host_params(p_i, p_f)
    scratch = pick_scratch(gridsum_partial)
    out = np.zeros(28)
    _lib.call("sky_nuclear_diagnostics", i32p(hi), len(hi), f64p(hf), len(hf), dptr(Field), f64p(np.ascontiguousarray(com)),
              dptr(scratch), _numel(scratch), f64p(out), stream_ptr())
    return com, out


def _store_com(com_d, com):
    if com_d is None:
        return
    import torch
    if isinstance(com_d, torch.Tensor):
        com_d.copy_(torch.from_numpy(com))
    else:
        com_d.copy_to_device(com)


class UTensorObservable:
    """compute_U_tensor(Field, d1fd1x, obs9, tensor_scratch, entmp, gridsum_partial, p_i_d, p_f_d, p_i_h)
    -> (3, 3): the isospin inertia tensor (observables.py:273-305)."""

    def __init__(self, theory_id):
        self.theory_id = theory_id

    def __call__(self, Field, d1fd1x, obs9, tensor_scratch, entmp, gridsum_partial, p_i_d, p_f_d, p_i_h=None):
        _, out = _nuclear_diag(self.theory_id, Field, gridsum_partial, p_i_h if p_i_h is not None else p_i_d, p_f_d)
        return _sym(out[0:6])


class _ComTensorObservable:
    """(Field, grid, d1fd1x, obs9, tensor_scratch, entmp, gridsum_partial, obs4, com_d, p_i_d, p_f_d, p_i_h)
    -> (3, 3), about the centre of mass, which is also written to com_d."""

    def __init__(self, theory_id):
        self.theory_id = theory_id

    def __call__(self, Field, grid, d1fd1x, obs9, tensor_scratch, entmp, gridsum_partial, obs4, com_d, p_i_d, p_f_d,
                 p_i_h=None):
        com, out = _nuclear_diag(self.theory_id, Field, gridsum_partial, p_i_h if p_i_h is not None else p_i_d,
                                 p_f_d)
        _store_com(com_d, com)
        return self.pick(out)


class VTensorObservable(_ComTensorObservable):
    """compute_V_tensor: the spin inertia tensor (observables.py:308-349)."""

    @staticmethod
    def pick(out):
        return _sym(out[6:12])


class WTensorObservable(_ComTensorObservable):
    """compute_W_tensor: the mixed inertia tensor (observables.py:352-393)."""

    @staticmethod
    def pick(out):
        return out[12:21].reshape(3, 3).copy()


class QuadrupoleTensorObservable(_ComTensorObservable):
    """compute_quadrupole_tensor: the baryon quadrupole tensor (observables.py:396-437)."""

    @staticmethod
    def pick(out):
        return _sym(out[21:27])


class DTermObservable:
    """compute_D_term(Field, grid, d1fd1x, en, entmp, gridsum_partial, obs4, tensor_scratch, com_d, p_i_d, p_f_d,
    p_i_h, p_f_h) -> float: -(2/5) E times the stress integral about the centre of mass
    (observables.py:440-487); en and entmp are left zeroed."""

    def __init__(self, theory_id):
        self.theory_id = theory_id

    def __call__(self, Field, grid, d1fd1x, en, entmp, gridsum_partial, obs4, tensor_scratch, com_d, p_i_d, p_f_d,
                 p_i_h=None, p_f_h=None):
        p_i = p_i_h if p_i_h is not None else p_i_d
        p_f = p_f_h if p_f_h is not None else p_f_d
        com, out = _nuclear_diag(self.theory_id, Field, gridsum_partial, p_i, p_f)
        _store_com(com_d, com)
        E = _total("sky_total_energy", self.theory_id, Field, en, entmp, gridsum_partial, p_i, p_f)
        return -(2.0 / 5.0) * E * float(out[27])
