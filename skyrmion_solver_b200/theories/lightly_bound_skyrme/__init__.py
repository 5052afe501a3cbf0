"""Lightly bound Skyrme model: theory package with the reference's submodules (params, kernels,
initial_config, observables, io, render_headless) backed by the sm_100a engine."""
from __future__ import annotations

from ..registry import TheorySpec
from . import initial_config, io, kernels, observables, params, render_headless

THEORY_SPEC = TheorySpec(
    name="Lightly bound Skyrme model",
    aliases=('Lightly bound Skyrme', 'Loosely bound Skyrme', 'Loosely bound Skyrme model'),
    import_path="skyrmion_solver_b200.theories.lightly_bound_skyrme",
    description="Lightly bound Skyrme model with the alpha (1 - sigma)^4 potential.",
    version="1.0",
)
SHORT_NAME = "lightly_bound"


def describe() -> None:
    print(THEORY_SPEC.name + ": " + THEORY_SPEC.description)
    params.describe()
