"""Nuclear Skyrme model: theory package with the reference's submodules (params, kernels,
initial_config, observables, io, render_headless) backed by the sm_100a engine."""
from __future__ import annotations

from ..registry import TheorySpec
from . import initial_config, io, kernels, observables, params, render_headless

THEORY_SPEC = TheorySpec(
    name="Nuclear Skyrme model",
    aliases=('Skyrme Model', '3D skyrmions', 'Skyrmions'),
    import_path="skyrmion_solver_b200.theories.nuclear_skyrme",
    description="Skyrmions in the 3D nuclear Skyrme model, with the standard pion mass potential.",
    version="1.0",
)
SHORT_NAME = "nuclear"


def describe() -> None:
    print(THEORY_SPEC.name + ": " + THEORY_SPEC.description)
    params.describe()
