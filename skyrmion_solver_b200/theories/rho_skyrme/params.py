"""Rho-meson Skyrme parameters (skyrmion_solver th/rho_skyrme/params.py).

Derived couplings: mpi = 2 m_pi/(e f_pi), mrho = 2 m_rho/(e f_pi), c_alpha = alpha e.
Device packing: p_f[8] = mpi, p_f[9] = mrho, p_f[10] = c_alpha.
"""
from __future__ import annotations

from dataclasses import dataclass

from ...core.params import Params as CoreParams
from ...core.params import ResolvedParams as CoreResolvedParams
from ...core.params import pack_device_params as pack_core_device_params
from .._common import ansatz_flags, ansatz_ints, core_values, pack


@dataclass(frozen=True)
class Params(CoreParams):
    number_total_fields: int = 13
    mass_pion: float = 138.0
    mass_rho: float = 775.0
    f_pi: float = 129.0
    e_skyrme: float = 1.0
    alpha: float = 0.0617
    mpi: float | None = None
    mrho: float | None = None
    c_alpha: float | None = None
    baryon_number: float = 1.0
    isospin_rotation: float = 0.0
    ansatz: str = "hedgehog"

    def resolved(self) -> "ResolvedParams":
        return ResolvedParams.from_params(self)


@dataclass(frozen=True)
class ResolvedParams(CoreResolvedParams):
    mass_pion: float
    mass_rho: float
    f_pi: float
    e_skyrme: float
    alpha: float
    mpi: float
    mrho: float
    c_alpha: float
    mpi_is_derived: bool
    mrho_is_derived: bool
    c_alpha_is_derived: bool
    baryon_number: float
    isospin_rotation: float
    ansatz_hedgehog: bool
    ansatz_rational_map: bool
    ansatz_uniform: bool

    @staticmethod
    def from_params(p: Params) -> "ResolvedParams":
        flags = ansatz_flags(p.ansatz)
        need = (p.mpi is None) or (p.mrho is None) or (p.c_alpha is None)
        if need and float(p.e_skyrme) == 0.0:
            raise ValueError("e_skyrme must be nonzero when deriving mpi, mrho, or c_alpha.")
        if need and float(p.f_pi) == 0.0:
            raise ValueError("f_pi must be nonzero when deriving mpi or mrho.")
        denom = float(p.e_skyrme) * float(p.f_pi)
        mpi = 2.0 * float(p.mass_pion) / denom if p.mpi is None else float(p.mpi)
        mrho = 2.0 * float(p.mass_rho) / denom if p.mrho is None else float(p.mrho)
        c_alpha = float(p.alpha) * float(p.e_skyrme) if p.c_alpha is None else float(p.c_alpha)
        return ResolvedParams(**core_values(p), mass_pion=float(p.mass_pion), mass_rho=float(p.mass_rho),
                              f_pi=float(p.f_pi), e_skyrme=float(p.e_skyrme), alpha=float(p.alpha), mpi=mpi,
                              mrho=mrho, c_alpha=c_alpha, mpi_is_derived=p.mpi is None,
                              mrho_is_derived=p.mrho is None, c_alpha_is_derived=p.c_alpha is None,
                              baryon_number=float(p.baryon_number), isospin_rotation=float(p.isospin_rotation),
                              **flags)


def default_params(**overrides) -> Params:
    return Params().with_(**overrides)


def pack_device_params(rp: ResolvedParams):
    return pack(rp, pack_core_device_params, ansatz_ints(rp),
                [rp.mpi, rp.mrho, rp.c_alpha, rp.baryon_number, rp.isospin_rotation])


def describe() -> None:
    print("Rho-meson Skyrme model: 13 components (phi0..3, rho_i^a at 4+3i+a); mpi, mrho, c_alpha = p_f[8..10].")
