"""Rho Skyrme model: theory package with the reference's submodules (params, kernels,
initial_config, observables, io, render_headless) backed by the sm_100a engine."""
from __future__ import annotations

from ..registry import TheorySpec
from . import initial_config, io, kernels, observables, params, render_headless

THEORY_SPEC = TheorySpec(
    name="Rho-Skyrme model",
    aliases=('Rho-Skyrme', 'Rho-skyrmions', 'Skyrmions with rho mesons'),
    import_path="skyrmion_solver_b200.theories.rho_skyrme",
    description="Skyrmions coupled to the rho meson (rho_i^a spatial components).",
    version="1.0",
)
SHORT_NAME = "rho"


def describe() -> None:
    print(THEORY_SPEC.name + ": " + THEORY_SPEC.description)
    params.describe()
