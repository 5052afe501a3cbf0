"""Theory registry with the reference's interface (skyrmion_solver th/registry.py:19-318)."""
from __future__ import annotations

import importlib
import pkgutil
from dataclasses import dataclass
from types import ModuleType
from typing import Dict


@dataclass(frozen=True)
class TheorySpec:
    name: str
    import_path: str
    description: str = ""
    version: str = "0.0"
    aliases: tuple = ()
    required_submodules: tuple = ("kernels", "initial_config", "observables")


_REGISTRY: Dict[str, TheorySpec] = {}


def register_theory(spec: TheorySpec) -> None:
    for k in [spec.name, *spec.aliases]:
        key = (k or "").strip().lower()
        if not key:
            raise ValueError("TheorySpec names must be non-empty")
        if key in _REGISTRY:
            raise ValueError(f"Theory '{key}' is already registered")
        _REGISTRY[key] = spec


def list_theories() -> tuple:
    return tuple(sorted({spec.name for spec in _REGISTRY.values()}))


def get_theory_spec(name: str) -> TheorySpec:
    key = (name or "").strip().lower()
    if key not in _REGISTRY:
        raise KeyError(f"Unknown theory '{name}'. Available: {list_theories()}")
    return _REGISTRY[key]


def load_theory(name: str) -> ModuleType:
    spec = get_theory_spec(name)
    mod = importlib.import_module(spec.import_path)
    for sub in spec.required_submodules:
        importlib.import_module(f"{spec.import_path}.{sub}")
    return mod


def describe_theory(name: str) -> None:
    spec = get_theory_spec(name)
    print(f"Theory: {spec.name}")
    print(f"Import path: {spec.import_path}")
    print(f"Version: {spec.version}")
    if spec.aliases:
        print("Aliases:", ", ".join(spec.aliases))
    if spec.description:
        print(f"Description: {spec.description}")


def print_theory_table() -> None:
    for spec in sorted({s for s in _REGISTRY.values()}, key=lambda s: s.name.lower()):
        print(f"{spec.name:<28} {spec.version:<6} {spec.description}")


def discover_theories(package: str = "skyrmion_solver_b200.theories") -> None:
    """Register every sub-package exposing THEORY_SPEC.  Unlike the reference
    (th/registry.py:302-305) an import failure is raised, not silently skipped."""
    pkg = importlib.import_module(package)
    for m in pkgutil.iter_modules(pkg.__path__):
        if not m.ispkg or m.name.startswith("_"):
            continue
        sub = importlib.import_module(f"{package}.{m.name}")
        spec = getattr(sub, "THEORY_SPEC", None)
        if isinstance(spec, TheorySpec):
            for k in [spec.name, *spec.aliases]:
                key = (k or "").strip().lower()
                if key and key not in _REGISTRY:
                    _REGISTRY[key] = spec
