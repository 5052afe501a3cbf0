"""Berger Skyrme model: theory package with the reference's submodules (params, kernels,
initial_config, observables, io, render_headless) backed by the sm_100a engine."""
from __future__ import annotations

from ..registry import TheorySpec
from . import initial_config, io, kernels, observables, params, render_headless

THEORY_SPEC = TheorySpec(
    name="Berger Skyrme model",
    aliases=('Berger Skyrme', 'Squashed sphere Skyrme', 'Berger skyrmions'),
    import_path="skyrmion_solver_b200.theories.berger_skyrme",
    description="Skyrmions with a Berger-sphere deformed target metric.",
    version="1.0",
)
SHORT_NAME = "berger"


def describe() -> None:
    print(THEORY_SPEC.name + ": " + THEORY_SPEC.description)
    params.describe()
