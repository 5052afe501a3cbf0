"""Time stepping with the reference's interface (skyrmion_solver ``core/integrator.py``).

``do_arrested_newton_flow`` keeps the reference's signature and schedule
(core/integrator.py:284-410).  When the gradient / RK4 kernels and the energy
routine are this library's, the whole step runs as one C-ABI call
(``sky_arrested_newton_step``); otherwise the schedule is driven from Python
with whatever launchables were passed.
"""
from __future__ import annotations

import ctypes

from .. import _lib
from .._lib import dptr, f64p, host_params, i32p, stream_ptr
from .launch import ArrestingCriteriaKernel, RK4FinalizeKernel, RK4StageKernel
from .utils import compute_max_field, launch_3d, pick_scratch, set_field_zero_kernel, _numel

do_rk4_step_kernel = RK4StageKernel()
do_rk4_kernel_no_constraint = RK4FinalizeKernel(-1, "do_rk4_kernel_no_constraint")
arresting_criteria_kernel = ArrestingCriteriaKernel()


def arresting_criteria(Velocity, EnergyGradient, en, entmp, gridsum_partial, p_i_d, p_i_h) -> float:
    """Lattice sum of the power V . EG (core/integrator.py:243-282), one fused launch with a
    compensated sum; leaves en and entmp zeroed, as the reference does."""
    hi, _ = host_params(p_i_h)
    scratch = pick_scratch(gridsum_partial)
    out = ctypes.c_double(0.0)
    _lib.call("sky_arresting_criteria", i32p(hi), len(hi), dptr(Velocity), dptr(EnergyGradient), None,
              dptr(scratch), _numel(scratch), ctypes.byref(out), stream_ptr())
    from .observables import _zero
    _zero(en, entmp)
    return float(out.value)


def make_do_gradient_step_kernel(do_gradient_step_point):
    """The reference builds gradient kernels from Numba device functions; this engine's
    gradient kernels are compiled CUDA, selected per theory (see each theory's kernels module)."""
    raise NotImplementedError(
        "custom per-site point functions are not JIT-compiled here; use a theory's "
        "kernels.do_gradient_step_kernel (nuclear, omega, coulomb, rho, berger, lightly_bound)")


def make_do_rk4_kernel(compute_norm_skyrme_field, project_orthogonal_skyrme_field):
    raise NotImplementedError(
        "custom norm / projection device functions are not JIT-compiled here; use a theory's "
        "kernels.do_rk4_kernel")


def do_arrested_newton_flow(Velocity, Field, d1fd1x, d2fd2x, EnergyGradient, k1, k2, k3, k4, l1, l2, l3, l4, Temp,
                            en, entmp, gridsum_partial, max_partial, p_i_d, p_f_d, p_i_h, p_f_h, prev_energy,
                            compute_energy, gradient_step_kernel, rk4_kernel, compute_norm=None,
                            do_norm_kernel=None):
    """One arrested-Newton RK4 step; returns (new_energy, err) (core/integrator.py:284-410)."""
    theory_id = getattr(gradient_step_kernel, "theory_id", None)
    fused = (theory_id is not None and getattr(rk4_kernel, "theory_id", None) == theory_id
             and getattr(compute_energy, "theory_id", None) == theory_id
             and (compute_norm is None or do_norm_kernel is None))
    if fused:
        hi, hf = host_params(p_i_h, p_f_h)
        scratch = pick_scratch(gridsum_partial, slots=2)
        e = ctypes.c_double(0.0)
        err = ctypes.c_double(0.0)
        _lib.call("sky_arrested_newton_step", theory_id, i32p(hi), len(hi), f64p(hf), len(hf), dptr(Velocity),
                  dptr(Field), dptr(EnergyGradient), dptr(k1), dptr(k2), dptr(k3), dptr(k4), dptr(l1), dptr(l2),
                  dptr(l3), dptr(l4), dptr(Temp), dptr(scratch), _numel(scratch), float(prev_energy),
                  ctypes.byref(e), ctypes.byref(err), stream_ptr())
        return float(e.value), float(err.value)

    grid3d, block3d = launch_3d(p_i_h, threads=(8, 8, 4))

    def normalize_field(target):
        if compute_norm is None or do_norm_kernel is None:
            return
        norm = compute_norm(target, en, entmp, gridsum_partial, p_i_d, p_i_h, p_f_d)
        do_norm_kernel[grid3d, block3d](target, norm, p_i_d)

    do_rk4_step_kernel[grid3d, block3d](k1, Velocity, Velocity, Temp, Field, Field, 0.0, p_i_d, p_f_d)
    normalize_field(Temp)
    gradient_step_kernel[grid3d, block3d](l1, Temp, d1fd1x, d2fd2x, EnergyGradient, p_i_d, p_f_d)
    do_rk4_step_kernel[grid3d, block3d](k2, Velocity, l1, Temp, Field, k1, 0.5, p_i_d, p_f_d)
    normalize_field(Temp)
    gradient_step_kernel[grid3d, block3d](l2, Temp, d1fd1x, d2fd2x, EnergyGradient, p_i_d, p_f_d)
    do_rk4_step_kernel[grid3d, block3d](k3, Velocity, l2, Temp, Field, k2, 0.5, p_i_d, p_f_d)
    normalize_field(Temp)
    gradient_step_kernel[grid3d, block3d](l3, Temp, d1fd1x, d2fd2x, EnergyGradient, p_i_d, p_f_d)
    do_rk4_step_kernel[grid3d, block3d](k4, Velocity, l3, Temp, Field, k3, 1.0, p_i_d, p_f_d)
    normalize_field(Temp)
    gradient_step_kernel[grid3d, block3d](l4, Temp, d1fd1x, d2fd2x, EnergyGradient, p_i_d, p_f_d)
    rk4_kernel[grid3d, block3d](Velocity, Field, k1, k2, k3, k4, l1, l2, l3, l4, p_i_d, p_f_d)
    normalize_field(Field)
    new_energy = compute_energy(Field, d1fd1x, en, entmp, gridsum_partial, p_i_d, p_f_d, p_i_h, p_f_h)
    if int(p_i_h[8]) and new_energy > prev_energy:
        set_field_zero_kernel[grid3d, block3d](Velocity, p_i_d)
    err = compute_max_field(EnergyGradient, max_partial, p_i_h)
    return new_energy, err
