"""Launchable kernel objects with the reference's Numba launch syntax.

The reference launches kernels as ``kernel[grid3d, block3d](*args)`` with 1-D
FP64 device arrays (e.g. core/integrator.py:382-398).  The objects below keep
that syntax and argument order; the launch geometry is chosen by the library
(the bracket configuration is accepted and ignored), and each call runs the
corresponding sm_100a kernel through the C ABI on the current torch stream.

Arguments may be torch CUDA tensors or any ``__cuda_array_interface__``
object (e.g. Numba device arrays).  ``p_i`` / ``p_f`` may be ``DeviceParams``
(host copy attached, no synchronisation), numpy arrays, or device arrays
(copied to the host once per call).
"""
from __future__ import annotations

import numpy as np

from .. import _lib
from .._lib import dptr, f64p, host_params, i32p, stream_ptr


class DeviceParams:
    """A packed parameter array resident on the device with its host copy.

    Acts as a device array (``__cuda_array_interface__``) while letting the
    launchers read the values without a device-to-host copy.
    """

    def __init__(self, host: np.ndarray, device=None):
        self.host = np.ascontiguousarray(host)
        if device is None:
            import torch
            device = torch.from_numpy(self.host.copy()).cuda()
        self.device = device

    @property
    def __cuda_array_interface__(self):
        return self.device.__cuda_array_interface__

    def copy_to_host(self):
        return self.host.copy()

    def __len__(self):
        return len(self.host)

    def __getitem__(self, i):
        return self.host[i]


class Launchable:
    """Base: ``kernel[grid, block]`` returns the kernel itself."""

    name = "kernel"

    def __getitem__(self, config):
        return self

    def _params(self, p_i, p_f=None):
        hi, hf = host_params(p_i, p_f)
        return hi, hf


class GradientKernel(Launchable):
    """do_gradient_step_kernel(l_out, Field, d1fd1x, d2fd2x, EnergyGradient, p_i, p_f)
    (core/integrator.py:37-46).  d1fd1x / d2fd2x are not touched."""

    def __init__(self, theory_id: int, name: str):
        self.theory_id = theory_id
        self.name = name

    def __call__(self, l_out, Field, d1fd1x, d2fd2x, EnergyGradient, p_i, p_f):
        hi, hf = self._params(p_i, p_f)
        _lib.call("sky_gradient_step", self.theory_id, i32p(hi), len(hi), f64p(hf), len(hf),
                  dptr(l_out), dptr(Field), dptr(EnergyGradient), stream_ptr())


class RK4StageKernel(Launchable):
    """do_rk4_step_kernel(k_out, Velocity, l_in, Temp, Field, k_prev, factor, p_i, p_f)
    (core/integrator.py:50-92)."""

    name = "do_rk4_step_kernel"

    def __call__(self, k_out, Velocity, l_in, Temp, Field, k_prev, factor, p_i, p_f):
        hi, hf = self._params(p_i, p_f)
        _lib.call("sky_rk4_stage", i32p(hi), len(hi), f64p(hf), len(hf), dptr(k_out), dptr(Velocity),
                  dptr(l_in), dptr(Temp), dptr(Field), dptr(k_prev), float(factor), stream_ptr())


class RK4FinalizeKernel(Launchable):
    """do_rk4_kernel(Velocity, Field, k1, k2, k3, k4, l1, l2, l3, l4, p_i, p_f)
    (core/integrator.py:94-177).  theory_id < 0 is the unconstrained variant."""

    def __init__(self, theory_id: int, name: str):
        self.theory_id = theory_id
        self.name = name

    def __call__(self, Velocity, Field, k1, k2, k3, k4, l1, l2, l3, l4, p_i, p_f):
        hi, hf = self._params(p_i, p_f)
        _lib.call("sky_rk4_finalize", self.theory_id, i32p(hi), len(hi), f64p(hf), len(hf), dptr(Velocity),
                  dptr(Field), dptr(k1), dptr(k2), dptr(k3), dptr(k4), dptr(l1), dptr(l2), dptr(l3), dptr(l4),
                  stream_ptr())


class DensityKernel(Launchable):
    """compute_energy_kernel / compute_skyrmion_number_kernel(en, Field, d1fd1x, p_i, p_f)."""

    def __init__(self, theory_id: int, mode: int, name: str):
        self.theory_id = theory_id
        self.mode = mode
        self.name = name

    def __call__(self, en, Field, d1fd1x, p_i, p_f):
        hi, hf = self._params(p_i, p_f)
        fn = "sky_energy_density" if self.mode == 0 else "sky_baryon_density"
        _lib.call(fn, self.theory_id, i32p(hi), len(hi), f64p(hf), len(hf), dptr(en), dptr(Field), stream_ptr())


class PotentialKernel(Launchable):
    """compute_potential_kernel(en, Field, p_i, p_f) (th/omega_skyrme/kernels.py:413-441)."""

    name = "compute_potential_kernel"

    def __call__(self, en, Field, p_i, p_f=None):
        hi, _ = self._params(p_i)
        _lib.call("sky_potential_density", i32p(hi), len(hi), dptr(en), dptr(Field), stream_ptr())


class RhoMesonKernel(Launchable):
    """compute_rho_meson_kernel(en, Field, p_i) (th/rho_skyrme/kernels.py:385-412); accumulates."""

    name = "compute_rho_meson_kernel"

    def __call__(self, en, Field, p_i):
        hi, _ = self._params(p_i)
        _lib.call("sky_rho_meson_density", i32p(hi), len(hi), dptr(en), dptr(Field), stream_ptr())


class ArrestingCriteriaKernel(Launchable):
    """arresting_criteria_kernel(Velocity, EnergyGradient, en, p_i) (core/integrator.py:213-241):
    en = per-site power V . EG."""

    name = "arresting_criteria_kernel"

    def __call__(self, Velocity, EnergyGradient, en, p_i):
        from .utils import reduction_scratch
        hi, _ = self._params(p_i)
        scratch = reduction_scratch()
        _lib.call("sky_arresting_criteria", i32p(hi), len(hi), dptr(Velocity), dptr(EnergyGradient), dptr(en),
                  dptr(scratch), scratch.numel(), None, stream_ptr())


class SetFieldZeroKernel(Launchable):
    """set_field_zero_kernel(Field, p_i) (core/utils.py:148-174)."""

    name = "set_field_zero_kernel"

    def __call__(self, Field, p_i):
        hi, _ = self._params(p_i)
        _lib.call("sky_set_field_zero", i32p(hi), len(hi), dptr(Field), stream_ptr())


class CreateGridKernel(Launchable):
    """create_grid_kernel(grid, p_i, p_f) (th/nuclear_skyrme/kernels.py:27-56)."""

    name = "create_grid_kernel"

    def __call__(self, grid, p_i, p_f):
        hi, hf = self._params(p_i, p_f)
        _lib.call("sky_create_grid", i32p(hi), len(hi), f64p(hf), len(hf), dptr(grid), stream_ptr())
