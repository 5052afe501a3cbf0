"""Simulation driver with the reference's interface (skyrmion_solver ``core/simulation.py:28-493``).

``Simulation(params, theory)`` owns the FP64 device buffers (torch CUDA tensors
in the reference's flattened SoA layout) and exposes the same attributes and
methods: ``initialize``, ``set_params``, ``observables``, ``compute_*_density``,
``step``, ``save_output``.  Buffers the engine never needs (the derivative
scratch ``d1fd1x`` / ``d2fd2x`` and the diagnostic tensors) are allocated on
first access only.
"""
from __future__ import annotations

import inspect
from pathlib import Path

import numpy as np

from .integrator import do_arrested_newton_flow, do_rk4_kernel_no_constraint
from .launch import DeviceParams
from .params import Params
from .utils import launch_3d, scratch_doubles, set_field_zero_kernel


def _torch():
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("skyrmion_b200 needs a CUDA device (sm_100a); none is visible")
    return torch


class Simulation:
    _LAZY = {
        "d1fd1x": lambda rp: rp.number_coordinates * rp.number_total_fields * rp.dim_grid,
        "d2fd2x": lambda rp: rp.number_coordinates ** 2 * rp.number_total_fields * rp.dim_grid,
        "obs4": lambda rp: 4 * rp.dim_grid,
        "obs9": lambda rp: 9 * rp.dim_grid,
        "tensor_scratch": lambda rp: rp.dim_grid,
        "com_d": lambda rp: 3,
    }

    def __init__(self, params, theory):
        self.theory = theory
        self.kernels = theory.kernels
        self.initial_config = theory.initial_config
        self.observables_mod = theory.observables
        self.threads3d = getattr(self.theory, "threads3d", (8, 8, 4))
        self.gradient_step_kernel = getattr(self.kernels, "do_gradient_step_kernel", None)
        if self.gradient_step_kernel is None:
            raise AttributeError("Theory kernels must provide do_gradient_step_kernel.")
        self.rk4_kernel = getattr(self.kernels, "do_rk4_kernel", None)
        if self.rk4_kernel is None:
            self.rk4_kernel = do_rk4_kernel_no_constraint
        self.set_params(params)
        torch = _torch()
        rp = self.rp
        dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev

        def arr(n):
            return torch.empty(int(n), dtype=torch.float64, device=dev)

        for name in ("Field", "Velocity", "EnergyGradient", "k1", "k2", "k3", "k4", "l1", "l2", "l3", "l4",
                     "Temp"):
            setattr(self, name, arr(rp.dim_fields))
        self.grid = arr(rp.number_coordinates * rp.dim_grid)
        self.en = torch.zeros(rp.dim_grid, dtype=torch.float64, device=dev)
        self.entmp = torch.zeros(rp.dim_grid, dtype=torch.float64, device=dev)
        self.gridsum_partial = torch.zeros(2 * scratch_doubles(), dtype=torch.float64, device=dev)
        self.max_partial = torch.zeros(scratch_doubles(), dtype=torch.float64, device=dev)

    def __getattr__(self, name):
        # lazily allocated buffers with the reference's sizes
        sizes = type(self)._LAZY
        if name in sizes and "rp" in self.__dict__:
            torch = _torch()
            buf = torch.zeros(int(sizes[name](self.rp)), dtype=torch.float64, device=self.device)
            setattr(self, name, buf)
            return buf
        raise AttributeError(name)

    # ------------------------------------------------------------------
    def set_params(self, p):
        """Resolve and pack the parameters (core/simulation.py:175-197)."""
        self.p = p
        self.rp = p.resolved() if isinstance(p, Params) else p
        p_i_h, p_f_h = self.theory.params.pack_device_params(self.rp)
        self.p_i_h = np.asarray(p_i_h, dtype=np.int32)
        self.p_f_h = np.asarray(p_f_h, dtype=np.float64)
        self.p_i_d = DeviceParams(self.p_i_h)
        self.p_f_d = DeviceParams(self.p_f_h)

    def initialize(self, init_config: dict | None = None):
        """Grid, zeroed Field / Velocity, then the theory's initializer (core/simulation.py:124-173)."""
        cfg = init_config or {}
        grid3d, block3d = launch_3d(self.p_i_h, threads=self.threads3d)
        self.kernels.create_grid_kernel[grid3d, block3d](self.grid, self.p_i_d, self.p_f_d)
        set_field_zero_kernel[grid3d, block3d](self.Field, self.p_i_d)
        set_field_zero_kernel[grid3d, block3d](self.Velocity, self.p_i_d)
        kw = dict(Velocity=self.Velocity, Field=self.Field, grid=self.grid, k1=self.k1, k2=self.k2, k3=self.k3,
                  k4=self.k4, l1=self.l1, l2=self.l2, l3=self.l3, l4=self.l4, Temp=self.Temp, p_i_d=self.p_i_d,
                  p_f_d=self.p_f_d, p_i_h=self.p_i_h, p_f_h=self.p_f_h, grid3d=grid3d, block3d=block3d, config=cfg)
        sig = inspect.signature(self.initial_config.initialize)
        if "d1fd1x" in sig.parameters:
            kw["d1fd1x"] = self.d1fd1x
        self.initial_config.initialize(**kw)
        _torch().cuda.synchronize()

    def observables(self):
        """Energy and baryon number (core/simulation.py:199-217)."""
        obs = {"energy": self.observables_mod.compute_energy(
            self.Field, None, self.en, self.entmp, self.gridsum_partial, self.p_i_d, self.p_f_d, self.p_i_h,
            self.p_f_h)}
        if hasattr(self.observables_mod, "compute_skyrmion_number"):
            obs["skyrmion_number"] = self.observables_mod.compute_skyrmion_number(
                self.Field, None, self.en, self.entmp, self.gridsum_partial, self.p_i_d, self.p_f_d, self.p_i_h)
        return obs

    def _launch(self):
        return launch_3d(self.p_i_h, threads=self.threads3d)

    def compute_energy_density(self):
        g, b = self._launch()
        self.kernels.compute_energy_kernel[g, b](self.en, self.Field, None, self.p_i_d, self.p_f_d)

    def compute_baryon_density(self):
        g, b = self._launch()
        self.kernels.compute_skyrmion_number_kernel[g, b](self.en, self.Field, None, self.p_i_d, self.p_f_d)

    def compute_potential_density(self):
        g, b = self._launch()
        self.kernels.compute_potential_kernel[g, b](self.en, self.Field, self.p_i_d, self.p_f_d)

    def compute_rho_meson_density(self):
        g, b = self._launch()
        self.kernels.compute_rho_meson_kernel[g, b](self.en, self.Field, self.p_i_d)

    def save_output(self, output_dir: str | None = None, precision: int = 32):
        """Write the theory's output bundle in the reference's ``.dat`` format
        (core/simulation.py:310-371): lattice metadata, the whole field, grid coordinates,
        field components and the energy and baryon densities (computed on the device)."""
        import inspect
        import os
        torch = _torch()
        if output_dir is None:
            output_dir = os.path.join(os.path.dirname(os.path.abspath(self.theory.io.__file__)), "results")
        os.makedirs(output_dir, exist_ok=True)
        self.compute_energy_density()
        h_energy = self.en.detach().cpu().numpy().copy()
        g, b = self._launch()
        self.kernels.compute_skyrmion_number_kernel[g, b](self.entmp, self.Field, None, self.p_i_d, self.p_f_d)
        torch.cuda.synchronize()
        h_baryon = self.entmp.detach().cpu().numpy().copy()
        if hasattr(self.kernels, "compute_potential_kernel"):
            self.compute_potential_density()
            torch.cuda.synchronize()
        kwargs = dict(output_dir=output_dir, h_Field=self.Field.detach().cpu().numpy(), h_EnergyDensity=h_energy,
                      h_BaryonDensity=h_baryon, h_OmegaDensity=self.en.detach().cpu().numpy(),
                      h_grid=self.grid.detach().cpu().numpy(), xlen=int(self.p_i_h[0]), ylen=int(self.p_i_h[1]),
                      zlen=int(self.p_i_h[2]), number_coordinates=int(self.p_i_h[4]),
                      number_total_fields=int(self.p_i_h[5]), precision=precision)
        accepted = set(inspect.signature(self.theory.io.output_data_bundle).parameters)
        self.theory.io.output_data_bundle(**{k: v for k, v in kwargs.items() if k in accepted})

    def compute_center_of_mass(self) -> np.ndarray:
        """Baryon-density centre of mass (core/simulation.py:390-403)."""
        return self.observables_mod.compute_center_of_mass(self.Field, self.grid, None, None, None, self.entmp,
                                                           self.gridsum_partial, self.p_i_d, self.p_f_d,
                                                           self.p_i_h)

    def compute_U_tensor(self) -> np.ndarray:
        """Isospin inertia tensor (core/simulation.py:420-433)."""
        return self.observables_mod.compute_U_tensor(self.Field, None, None, None, self.entmp, self.gridsum_partial,
                                                     self.p_i_d, self.p_f_d, self.p_i_h)

    def _com_tensor(self, fn):
        return fn(self.Field, self.grid, None, None, None, self.entmp, self.gridsum_partial, None, self.com_d,
                  self.p_i_d, self.p_f_d, self.p_i_h)

    def compute_V_tensor(self) -> np.ndarray:
        """Spin inertia tensor (core/simulation.py:435-448)."""
        return self._com_tensor(self.observables_mod.compute_V_tensor)

    def compute_W_tensor(self) -> np.ndarray:
        """Mixed inertia tensor (core/simulation.py:450-463)."""
        return self._com_tensor(self.observables_mod.compute_W_tensor)

    def compute_quadrupole_tensor(self) -> np.ndarray:
        """Baryon quadrupole tensor (core/simulation.py:465-478)."""
        return self._com_tensor(self.observables_mod.compute_quadrupole_tensor)

    def compute_D_term(self) -> float:
        """Monopole D-term (core/simulation.py:480-500)."""
        return self.observables_mod.compute_D_term(self.Field, self.grid, None, self.en, self.entmp,
                                                   self.gridsum_partial, None, None, self.com_d, self.p_i_d,
                                                   self.p_f_d, self.p_i_h, self.p_f_h)

    def compute_rms_radius(self) -> float:
        """Centre-of-mass RMS radius (core/simulation.py:405-418); the centre of mass lands in com_d."""
        return self.observables_mod.compute_rms_radius(self.Field, self.grid, None, self.en, self.entmp,
                                                       self.gridsum_partial, None, None, self.com_d, self.p_i_d,
                                                       self.p_f_d, self.p_i_h)

    def step(self, prev_energy: float):
        """One arrested-Newton / RK4 step; returns (new_energy, err) (core/simulation.py:287-308)."""
        compute_norm = getattr(self.observables_mod, "compute_norm", None)
        do_norm_kernel = getattr(self.kernels, "do_norm_kernel", None)
        return do_arrested_newton_flow(
            self.Velocity, self.Field, None, None, self.EnergyGradient, self.k1, self.k2, self.k3, self.k4,
            self.l1, self.l2, self.l3, self.l4, self.Temp, self.en, self.entmp, self.gridsum_partial,
            self.max_partial, self.p_i_d, self.p_f_d, self.p_i_h, self.p_f_h, prev_energy,
            self.observables_mod.compute_energy, self.gradient_step_kernel, self.rk4_kernel,
            compute_norm=compute_norm, do_norm_kernel=do_norm_kernel)

    def save_state(self, output_dir: str | None = None):
        """Snapshot of the state (field, velocity, densities, parameters) as ``state.npz``; the
        reference-format text bundle is ``save_output``."""
        out = Path(output_dir or "results")
        out.mkdir(parents=True, exist_ok=True)
        C = int(self.p_i_h[5])
        dims = tuple(int(v) for v in self.p_i_h[:3])
        self.compute_energy_density()
        ed = self.en.cpu().numpy().reshape(dims)
        self.compute_baryon_density()
        bd = self.en.cpu().numpy().reshape(dims)
        self.en.zero_()
        np.savez(out / "state.npz", Field=self.Field.cpu().numpy().reshape((C,) + dims),
                 Velocity=self.Velocity.cpu().numpy().reshape((C,) + dims), EnergyDensity=ed,
                 BaryonDensity=bd, p_i=self.p_i_h, p_f=self.p_f_h)

    def print_instructions(self):
        if hasattr(self.theory, "print_instructions"):
            self.theory.print_instructions()
        else:
            print("No specific instructions available for this theory.")
