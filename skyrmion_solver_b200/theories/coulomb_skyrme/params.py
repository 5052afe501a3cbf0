"""Coulomb Skyrme parameters (skyrmion_solver th/coulomb_skyrme/params.py).

Derived couplings: mass = 2 m_pi / (g f_pi), kappa = g^2 e^2 / 2.
Device packing: p_i[11] = number_skyrme_fields, p_f[8] = mass, p_f[9] = kappa.
"""
from __future__ import annotations

from dataclasses import dataclass

from ...core.params import Params as CoreParams
from ...core.params import ResolvedParams as CoreResolvedParams
from ...core.params import pack_device_params as pack_core_device_params
from .._common import ansatz_flags, ansatz_ints, core_values, pack


@dataclass(frozen=True)
class Params(CoreParams):
    number_total_fields: int = 5
    number_skyrme_fields: int = 4
    f_pi: float = 105.9
    m_pi: float = 138.0
    g: float = 4.0
    e: float = 0.302822
    mass: float | None = None
    kappa: float | None = None
    baryon_number: float = 1.0
    isospin_rotation: float = 0.0
    ansatz: str = "hedgehog"

    def resolved(self) -> "ResolvedParams":
        return ResolvedParams.from_params(self)


@dataclass(frozen=True)
class ResolvedParams(CoreResolvedParams):
    number_skyrme_fields: int
    f_pi: float
    m_pi: float
    g: float
    e: float
    mass: float
    kappa: float
    baryon_number: float
    isospin_rotation: float
    ansatz_hedgehog: bool
    ansatz_rational_map: bool
    ansatz_uniform: bool

    @staticmethod
    def from_params(p: Params) -> "ResolvedParams":
        flags = ansatz_flags(p.ansatz)
        if float(p.g) == 0.0:
            raise ValueError("g must be nonzero when deriving mass = 2 m_pi / (g f_pi).")
        if float(p.f_pi) == 0.0:
            raise ValueError("f_pi must be nonzero when deriving mass = 2 m_pi / (g f_pi).")
        mass = 2.0 * float(p.m_pi) / (float(p.g) * float(p.f_pi)) if p.mass is None else p.mass
        kappa = float(p.g) * float(p.g) * float(p.e) * float(p.e) / 2.0 if p.kappa is None else p.kappa
        return ResolvedParams(**core_values(p), number_skyrme_fields=int(p.number_skyrme_fields),
                              f_pi=float(p.f_pi), m_pi=float(p.m_pi), g=float(p.g), e=float(p.e), mass=mass,
                              kappa=kappa, baryon_number=float(p.baryon_number),
                              isospin_rotation=float(p.isospin_rotation), **flags)


def default_params(**overrides) -> Params:
    return Params().with_(**overrides)


def pack_device_params(rp: ResolvedParams):
    return pack(rp, pack_core_device_params, [rp.number_skyrme_fields] + ansatz_ints(rp),
                [rp.mass, rp.kappa, rp.baryon_number, rp.isospin_rotation])


def describe() -> None:
    print("Coulomb Skyrme model: 5 components (phi0..3, A0); mass = p_f[8], kappa = p_f[9].")
