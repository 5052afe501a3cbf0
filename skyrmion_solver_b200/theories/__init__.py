"""Theory discovery and loading (mirrors skyrmion_solver.theories)."""
from __future__ import annotations

from .registry import (TheorySpec, describe_theory, discover_theories, get_theory_spec, list_theories,
                       load_theory, print_theory_table, register_theory)

discover_theories()

SHORT_NAMES = {
    "nuclear": "nuclear_skyrme", "omega": "omega_skyrme", "coulomb": "coulomb_skyrme", "rho": "rho_skyrme",
    "berger": "berger_skyrme", "lightly_bound": "lightly_bound_skyrme",
}


def by_short_name(short: str):
    import importlib
    return importlib.import_module(f"{__name__}.{SHORT_NAMES[short]}")


def list():  # noqa: A001 - same name as the reference's helper
    return list_theories()


def print_description(name: str) -> None:
    describe_theory(name)


def print_table() -> None:
    print_theory_table()
