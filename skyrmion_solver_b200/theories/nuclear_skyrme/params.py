"""Nuclear (pion-only) Skyrme parameters (skyrmion_solver th/nuclear_skyrme/params.py:19-245).

Device packing: p_f[8] = mpi, p_f[9] = kappa (the kernels' coupling slots).
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
    baryon_number: float = 1.0
    isospin_rotation: float = 0.0
    ansatz: str = "hedgehog"

    def resolved(self) -> "ResolvedParams":
        return ResolvedParams.from_params(self)


@dataclass(frozen=True)
class ResolvedParams(CoreResolvedParams):
    mpi: float
    kappa: float
    baryon_number: float
    isospin_rotation: float
    ansatz_hedgehog: bool
    ansatz_rational_map: bool
    ansatz_uniform: bool

    @staticmethod
    def from_params(p: Params) -> "ResolvedParams":
        return ResolvedParams(**core_values(p), mpi=float(p.mpi), kappa=float(p.kappa),
                              baryon_number=float(p.baryon_number), isospin_rotation=float(p.isospin_rotation),
                              **ansatz_flags(p.ansatz))


def default_params(**overrides) -> Params:
    return Params().with_(**overrides)


def pack_device_params(rp: ResolvedParams):
    return pack(rp, pack_core_device_params, ansatz_ints(rp),
                [rp.mpi, rp.kappa, rp.baryon_number, rp.isospin_rotation])


def describe() -> None:
    print("Nuclear Skyrme model: 4 components (sigma, pi1, pi2, pi3); couplings mpi = p_f[8], kappa = p_f[9].")
