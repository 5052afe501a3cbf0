"""Kernels of the Lightly bound Skyrme model (th/lightly_bound_skyrme/kernels.py in skyrmion_solver), as sm_100a launchables.

Same attribute names and launch syntax as the reference module; see
``skyrmion_solver_b200.core.launch`` for the argument conventions.
"""
from ...core.launch import CreateGridKernel, DensityKernel, GradientKernel, PotentialKernel, RhoMesonKernel, \
    RK4FinalizeKernel

THEORY_ID = 5

create_grid_kernel = CreateGridKernel()
do_gradient_step_kernel = GradientKernel(THEORY_ID, "do_gradient_step_kernel")
do_rk4_kernel = RK4FinalizeKernel(THEORY_ID, "do_rk4_kernel")
compute_energy_kernel = DensityKernel(THEORY_ID, 0, "compute_energy_kernel")
compute_skyrmion_number_kernel = DensityKernel(THEORY_ID, 1, "compute_skyrmion_number_kernel")
