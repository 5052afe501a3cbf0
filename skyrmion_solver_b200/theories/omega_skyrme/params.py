"""Omega-meson Skyrme parameters (skyrmion_solver th/omega_skyrme/params.py).

Derived couplings: mass = m_pi / m_omega, c_omega = m_omega * beta_omega / f_pi.
Device packing: p_i[11] = number_skyrme_fields, p_f[8] = mass, p_f[9] = c_omega.
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
    f_pi: float = 186.0
    m_pi: float = 138.0
    m_omega: float = 782.0
    beta_omega: float = 8.253
    mass: float | None = None
    c_omega: float | None = None
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
    m_omega: float
    beta_omega: float
    mass: float
    c_omega: float
    baryon_number: float
    isospin_rotation: float
    ansatz_hedgehog: bool
    ansatz_rational_map: bool
    ansatz_uniform: bool

    @staticmethod
    def from_params(p: Params) -> "ResolvedParams":
        flags = ansatz_flags(p.ansatz)
        if float(p.m_omega) == 0.0:
            raise ValueError("m_omega must be nonzero when deriving mass = m_pi / m_omega.")
        if float(p.f_pi) == 0.0:
            raise ValueError("f_pi must be nonzero when deriving c_omega = m_omega * beta_omega / f_pi.")
        mass = float(p.m_pi) / float(p.m_omega) if p.mass is None else p.mass
        c_omega = float(p.m_omega) * float(p.beta_omega) / float(p.f_pi) if p.c_omega is None else p.c_omega
        return ResolvedParams(**core_values(p), number_skyrme_fields=int(p.number_skyrme_fields),
                              f_pi=float(p.f_pi), m_pi=float(p.m_pi), m_omega=float(p.m_omega),
                              beta_omega=float(p.beta_omega), mass=mass, c_omega=c_omega,
                              baryon_number=float(p.baryon_number), isospin_rotation=float(p.isospin_rotation),
                              **flags)


def default_params(**overrides) -> Params:
    return Params().with_(**overrides)


def pack_device_params(rp: ResolvedParams):
    return pack(rp, pack_core_device_params, [rp.number_skyrme_fields] + ansatz_ints(rp),
                [rp.mass, rp.c_omega, rp.baryon_number, rp.isospin_rotation])


def describe() -> None:
    print("Omega-meson Skyrme model: 5 components (phi0..3, omega); mass = p_f[8], c_omega = p_f[9].")
