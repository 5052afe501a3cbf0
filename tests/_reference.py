"""The reference package, installed under baseline/_ref, for runs of its own code on a GPU.

``python -m pip install --no-index --no-build-isolation --no-deps --find-links
/opt/wheelhouse --target baseline/_ref <reference checkout>`` installs the
unmodified skyrmion_solver package (v1.0.2) next to this repository; it travels
with the repository to the GPU machine.  Its theory packages import their
OpenGL viewer (``render_gl``) from ``__init__``, so the core modules and each
theory's ``params``, ``kernels``, ``observables`` and ``initial_config`` are
imported here as sub-modules of bare package objects, without the viewer; no
graphics library is loaded.  Numba compiles the reference's kernels for the
GPU it finds (its built-in CUDA target emits PTX that the driver compiles for
the device).
"""
from __future__ import annotations

import importlib
import os
import sys
import types

ROOT = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "baseline", "_ref")

THEORY_DIRS = {
    "nuclear": "nuclear_skyrme",
    "omega": "omega_skyrme",
    "coulomb": "coulomb_skyrme",
    "rho": "rho_skyrme",
    "berger": "berger_skyrme",
    "lightly_bound": "lightly_bound_skyrme",
}


def available() -> bool:
    return os.path.isdir(os.path.join(ROOT, "skyrmion_solver", "core"))


def load(names=("omega",)):
    """(theory namespaces by short name, the reference's Simulation class, its core params module)."""
    if not available():
        raise RuntimeError(f"the reference is not installed under {ROOT}")
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    import skyrmion_solver  # noqa: F401  (empty package __init__)
    th_dir = os.path.join(ROOT, "skyrmion_solver", "theories")
    if "skyrmion_solver.theories" not in sys.modules or not hasattr(sys.modules["skyrmion_solver.theories"],
                                                                       "_viewer_free"):
        pkg = types.ModuleType("skyrmion_solver.theories")
        pkg.__path__ = [th_dir]
        pkg._viewer_free = True
        sys.modules["skyrmion_solver.theories"] = pkg
        importlib.import_module("skyrmion_solver.theories.registry")
    theories = {}
    for short in names:
        name = "skyrmion_solver.theories." + THEORY_DIRS[short]
        if name not in sys.modules:
            sub = types.ModuleType(name)
            sub.__path__ = [os.path.join(th_dir, THEORY_DIRS[short])]
            sys.modules[name] = sub
        ns = types.SimpleNamespace()
        for part in ("params", "kernels", "observables", "initial_config"):
            setattr(ns, part, importlib.import_module(name + "." + part))
        theories[short] = ns
    sim_mod = importlib.import_module("skyrmion_solver.core.simulation")
    params_mod = importlib.import_module("skyrmion_solver.core.params")
    return theories, sim_mod.Simulation, params_mod
