"""Coulomb Skyrme model: theory package with the reference's submodules (params, kernels,
initial_config, observables, io, render_headless) backed by the sm_100a engine."""
from __future__ import annotations

from ..registry import TheorySpec
from . import initial_config, io, kernels, observables, params, render_headless

THEORY_SPEC = TheorySpec(
    name="Coulomb-Skyrme model",
    aliases=('Coulomb Skyrme', 'Maxwell Skyrme'),
    import_path="skyrmion_solver_b200.theories.coulomb_skyrme",
    description="Skyrmions with an electrostatic A0 field (Coulomb interaction).",
    version="1.0",
)
SHORT_NAME = "coulomb"


def describe() -> None:
    print(THEORY_SPEC.name + ": " + THEORY_SPEC.description)
    params.describe()
