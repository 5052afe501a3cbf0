"""Berger-deformed Skyrme parameters (skyrmion_solver th/berger_skyrme/params.py).

Device packing: p_f[8] = mpi, p_f[9] = kappa, p_f[12] = alpha.
"""
from __future__ import annotations

from dataclasses import dataclass

from ...core.params import Params as CoreParams
from ...core.params import ResolvedParams as CoreResolvedParams
from ...core.params import pack_device_params as pack_core_device_params
from .._common import ansatz_flags, ansatz_ints, core_values, pack


@dataclass(frozen=True)
class Params(CoreParams):
    number_total_fields: int = 4
    mpi: float = 1.0
    kappa: float = 1.0
    alpha: float = 1.0
    baryon_number: float = 1.0
    isospin_rotation: float = 0.0
    ansatz: str = "hedgehog"

    def resolved(self) -> "ResolvedParams":
        return ResolvedParams.from_params(self)


@dataclass(frozen=True)
class ResolvedParams(CoreResolvedParams):
    mpi: float
    kappa: float
    alpha: float
    baryon_number: float
    isospin_rotation: float
    ansatz_hedgehog: bool
    ansatz_rational_map: bool
    ansatz_uniform: bool

    @staticmethod
    def from_params(p: Params) -> "ResolvedParams":
        return ResolvedParams(**core_values(p), mpi=float(p.mpi), kappa=float(p.kappa), alpha=float(p.alpha),
                              baryon_number=float(p.baryon_number), isospin_rotation=float(p.isospin_rotation),
                              **ansatz_flags(p.ansatz))


def default_params(**overrides) -> Params:
    return Params().with_(**overrides)


def pack_device_params(rp: ResolvedParams):
    return pack(rp, pack_core_device_params, ansatz_ints(rp),
                [rp.mpi, rp.kappa, rp.baryon_number, rp.isospin_rotation, rp.alpha])


def describe() -> None:
    print("Berger Skyrme model: 4 components; mpi = p_f[8], kappa = p_f[9], alpha = p_f[12].")
