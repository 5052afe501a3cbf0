"""Generate golden vectors by running the reference skyrmion_solver on the CPU.

The reference ships only Numba-CUDA kernels, so they are executed here under
Numba's CUDA simulator (``NUMBA_ENABLE_CUDASIM=1``).  This script is the only
place in the repository that imports the reference; it runs in the build
container (where the reference source tree is mounted) and writes small
``.npz`` fixtures that travel with the tests.  The GPU box never runs it.

Two things are needed to run the reference headless:

* The theory packages' ``__init__`` modules import the OpenGL viewer.  They are
  never executed: each theory package is pre-registered in ``sys.modules`` as a
  bare package object whose ``__path__`` points at the reference directory, so
  ``<theory>.params``, ``.kernels``, ``.observables`` load on their own.  No
  graphics module is imported or stubbed.
* Numba's simulator swaps the ``cuda`` global of a device function's module in
  and out on every device-function call (``swapped_cuda_module``).  Its
  per-CUDA-thread Python threads race on that swap (one thread's exit restores
  the real module while another is mid-call).  The patch below makes the swap
  idempotent during a launch and restores the module globals once, after the
  launch.  It changes scheduling only, never arithmetic.

Usage::

    python tests/golden/make_golden.py nuclear omega coulomb rho berger lightly_bound

Each theory writes ``tests/golden/<theory>.npz``.  Cost is about 30 s per
arrested-Newton step at 12x11x10 sites for C=4 (the simulator runs every CUDA
thread as a Python thread), so theories are best run as parallel processes.
"""
from __future__ import annotations

import os
import sys
import time
import types
import importlib
from contextlib import contextmanager

import numpy as np

REFERENCE_ROOT = os.environ.get("SKY_REFERENCE_ROOT", "/root/reference")
HERE = os.path.dirname(os.path.abspath(__file__))

THEORY_DIRS = {
    "nuclear": "nuclear_skyrme",
    "omega": "omega_skyrme",
    "coulomb": "coulomb_skyrme",
    "rho": "rho_skyrme",
    "berger": "berger_skyrme",
    "lightly_bound": "lightly_bound_skyrme",
}


def _patch_simulator():
    import numba.cuda.simulator.kernel as simk
    import numba.cuda.simulator.kernelapi as simapi

    touched = {}

    @contextmanager
    def swap_once(fn, fake_cuda_module):
        from numba import cuda
        g = fn.__globals__
        entry = touched.get(id(g))
        if entry is None:
            names = [k for k, v in g.items()
                     if v is cuda or isinstance(v, simapi.FakeCUDAModule)]
            entry = touched[id(g)] = (g, names)
        for k in entry[1]:
            g[k] = fake_cuda_module
        yield

    orig_call = simk.FakeCUDAKernel.__call__

    def call(self, *args):
        if self._device:
            return orig_call(self, *args)
        try:
            return orig_call(self, *args)
        finally:
            from numba import cuda
            for g, names in touched.values():
                for k in names:
                    g[k] = cuda
            touched.clear()

    simk.swapped_cuda_module = swap_once
    simk.FakeCUDAKernel.__call__ = call


def load_reference():
    """Import the reference core and theory sub-modules without their GL viewer."""
    os.environ["NUMBA_ENABLE_CUDASIM"] = "1"
    if REFERENCE_ROOT not in sys.path:
        sys.path.insert(0, REFERENCE_ROOT)
    _patch_simulator()
    import skyrmion_solver  # noqa: F401  (empty package __init__)
    th_dir = os.path.join(REFERENCE_ROOT, "skyrmion_solver", "theories")
    pkg = types.ModuleType("skyrmion_solver.theories")
    pkg.__path__ = [th_dir]
    sys.modules["skyrmion_solver.theories"] = pkg
    # registry has no GL dependency; load it so TheorySpec exists if needed
    importlib.import_module("skyrmion_solver.theories.registry")
    theories = {}
    for short, d in THEORY_DIRS.items():
        name = "skyrmion_solver.theories." + d
        sub = types.ModuleType(name)
        sub.__path__ = [os.path.join(th_dir, d)]
        sys.modules[name] = sub
        ns = types.SimpleNamespace()
        for part in ("params", "kernels", "observables"):
            setattr(ns, part, importlib.import_module(name + "." + part))
        ns.initial_config = types.SimpleNamespace(initialize=lambda **kw: None)
        theories[short] = ns
    sim_mod = importlib.import_module("skyrmion_solver.core.simulation")
    return theories, sim_mod.Simulation


# ---------------------------------------------------------------------------
# inputs
# ---------------------------------------------------------------------------
DIMS = (12, 11, 10)
SPACING = (0.2, 0.18, 0.22)


def theory_params(short, mod, **overrides):
    common = dict(xlen=DIMS[0], ylen=DIMS[1], zlen=DIMS[2],
                  lsx=SPACING[0], lsy=SPACING[1], lsz=SPACING[2],
                  xsize=SPACING[0] * (DIMS[0] - 1), ysize=SPACING[1] * (DIMS[1] - 1),
                  zsize=SPACING[2] * (DIMS[2] - 1),
                  time_step=0.02, killkinen=True, newtonflow=True, unit_length=True)
    extra = {
        "nuclear": dict(mpi=0.8, kappa=1.3),
        "omega": dict(),
        "coulomb": dict(),
        "rho": dict(mpi=0.586, mrho=3.29, c_alpha=0.2256, time_step=0.01),
        "berger": dict(mpi=0.9, kappa=1.1, alpha=1.3),
        "lightly_bound": dict(mpi=0.7, alpha=0.3),
    }[short]
    common.update(extra)
    common.update(overrides)
    return mod.params.default_params(**common)


def make_inputs(C, seed):
    rng = np.random.default_rng(seed)
    X, Y, Z = DIMS
    hx, hy, hz = SPACING
    xs = (np.arange(X) - (X - 1) / 2.0) * hx
    ys = (np.arange(Y) - (Y - 1) / 2.0) * hy
    zs = (np.arange(Z) - (Z - 1) / 2.0) * hz
    x, y, z = np.meshgrid(xs, ys, zs, indexing="ij")
    r = np.sqrt(x * x + y * y + z * z)
    f = np.pi * np.exp(-r / 0.8)
    rs = np.where(r > 0, r, 1.0)
    F = np.zeros((C, X, Y, Z))
    F[0] = np.cos(f)
    F[1] = np.sin(f) * x / rs
    F[2] = np.sin(f) * y / rs
    F[3] = np.sin(f) * z / rs
    F[:4] += rng.uniform(-0.02, 0.02, size=(4, X, Y, Z))
    F[:4] /= np.sqrt((F[:4] ** 2).sum(axis=0))
    for a in range(4, C):
        k = a - 3
        F[a] = 0.3 * np.exp(-r * r) * np.cos(k * x + 0.5 * y - 0.3 * k * z) \
            + rng.uniform(-0.01, 0.01, size=(X, Y, Z))
    V = rng.uniform(-1e-2, 1e-2, size=(C, X, Y, Z))
    T = F + rng.uniform(-0.05, 0.05, size=(C, X, Y, Z))  # off-sphere gradient input
    return F, V, T


def run(short, Simulation, th, nsteps=3):
    from numba import cuda
    from skyrmion_solver.core.utils import launch_3d
    p = theory_params(short, th)
    sim = Simulation(p, th)
    C = int(sim.p_i_h[5])
    F, V, T = make_inputs(C, seed=1234 + list(THEORY_DIRS).index(short))
    out = dict(p_i=np.asarray(sim.p_i_h), p_f=np.asarray(sim.p_f_h),
               field0=F, velocity0=V, temp_in=T)
    shp = (C,) + DIMS
    grid3d, block3d = launch_3d(sim.p_i_h, threads=(8, 8, 4))

    # standalone gradient kernel on an off-sphere field
    sim.Temp.copy_to_device(T.ravel())
    sim.gradient_step_kernel[grid3d, block3d](sim.l1, sim.Temp, sim.d1fd1x, sim.d2fd2x,
                                              sim.EnergyGradient, sim.p_i_d, sim.p_f_d)
    cuda.synchronize()
    out["grad_eg"] = sim.EnergyGradient.copy_to_host().reshape(shp)
    out["grad_l"] = sim.l1.copy_to_host().reshape(shp)

    sim.Field.copy_to_device(F.ravel())
    sim.Velocity.copy_to_device(V.ravel())

    # densities written into en by the per-site kernels
    sim.compute_energy_density()
    out["energy_density0"] = sim.en.copy_to_host().reshape(DIMS)
    sim.compute_baryon_density()
    out["baryon_density0"] = sim.en.copy_to_host().reshape(DIMS)
    if hasattr(th.kernels, "compute_potential_kernel"):
        sim.compute_potential_density()
        out["potential_density0"] = sim.en.copy_to_host().reshape(DIMS)
    if hasattr(th.kernels, "compute_rho_meson_kernel"):
        sim.en[:] = 0.0
        sim.compute_rho_meson_density()
        out["rho_meson_density0"] = sim.en.copy_to_host().reshape(DIMS)
    sim.en[:] = 0.0

    obs = sim.observables()
    out["energy0"] = np.float64(obs["energy"])
    out["baryon0"] = np.float64(obs.get("skyrmion_number", np.nan))

    prevs = [1e300, -1e300, None]
    energies, errs = [], []
    for s in range(nsteps):
        prev = prevs[s] if s < len(prevs) and prevs[s] is not None else energies[-1]
        t0 = time.time()
        e, err = sim.step(prev)
        print(f"[{short}] step {s}: E={e!r} err={err!r} ({time.time() - t0:.1f}s)", flush=True)
        energies.append(e)
        errs.append(err)
        out[f"prev{s}"] = np.float64(prev)
        out[f"field{s + 1}"] = sim.Field.copy_to_host().reshape(shp)
        out[f"velocity{s + 1}"] = sim.Velocity.copy_to_host().reshape(shp)
        out[f"eg{s + 1}"] = sim.EnergyGradient.copy_to_host().reshape(shp)
        if s == 0:
            for nm in ("k1", "k2", "k3", "k4", "l1", "l2", "l3", "l4", "Temp"):
                out[f"{nm}_1"] = getattr(sim, nm).copy_to_host().reshape(shp)
    out["energies"] = np.array(energies)
    out["errs"] = np.array(errs)
    obs = sim.observables()
    out["energy_final"] = np.float64(obs["energy"])
    out["baryon_final"] = np.float64(obs.get("skyrmion_number", np.nan))
    path = os.path.join(HERE, f"{short}.npz")
    np.savez_compressed(path, **out)
    print(f"[{short}] wrote {path}", flush=True)


def main(argv):
    names = argv or list(THEORY_DIRS)
    theories, Simulation = load_reference()
    for n in names:
        run(n, Simulation, theories[n])


if __name__ == "__main__":
    main(sys.argv[1:])
