"""Omega Skyrme model: theory package with the reference's submodules (params, kernels,
initial_config, observables, io, render_headless) backed by the sm_100a engine."""
from __future__ import annotations

from ..registry import TheorySpec
from . import initial_config, io, kernels, observables, params, render_headless

THEORY_SPEC = TheorySpec(
    name="Omega-Skyrme model",
    aliases=('Omega-Skyrme', 'Omega-meson model', 'Omega-meson Skyrme', 'Omega-sigma model'),
    import_path="skyrmion_solver_b200.theories.omega_skyrme",
    description="Skyrmions coupled to the omega meson (omega0 sourced by the baryon density).",
    version="1.0",
)
SHORT_NAME = "omega"


def describe() -> None:
    print(THEORY_SPEC.name + ": " + THEORY_SPEC.description)
    params.describe()
