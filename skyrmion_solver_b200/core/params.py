"""Core parameters: the reference's user-facing dataclasses and the packed
``p_i`` / ``p_f`` device ABI (skyrmion_solver ``core/params.py:15-267``).

The field names, defaults, derivations (h = size/(len-1), dt = courant * lsx)
and the positional packing are the reference's interface and are kept as is so
that existing parameter code runs unchanged.
"""
from __future__ import annotations

from dataclasses import dataclass, fields, replace

import numpy as np


@dataclass(frozen=True)
class Params:
    """User-facing core parameters shared by all theories (core/params.py:15-110)."""

    xlen: int = 64
    ylen: int = 64
    zlen: int = 64
    halo: int = 2
    number_coordinates: int = 3
    number_total_fields: int = 3
    xsize: float = 10.0
    ysize: float = 10.0
    zsize: float = 10.0
    lsx: float | None = None
    lsy: float | None = None
    lsz: float | None = None
    courant: float = 0.2
    time_step: float | None = None
    killkinen: bool = True
    newtonflow: bool = True
    unit_length: bool = True

    def with_(self, **kwargs) -> "Params":
        return replace(self, **kwargs)

    def resolved(self) -> "ResolvedParams":
        return ResolvedParams.from_params(self)


@dataclass(frozen=True)
class ResolvedParams:
    """Solver-ready parameters (core/params.py:112-226)."""

    xlen: int
    ylen: int
    zlen: int
    halo: int
    number_coordinates: int
    number_total_fields: int
    dim_grid: int
    dim_fields: int
    killkinen: int
    newtonflow: int
    unit_length: int
    xsize: float
    ysize: float
    zsize: float
    lsx: float
    lsy: float
    lsz: float
    grid_volume: float
    time_step: float

    @staticmethod
    def core_values(p: Params) -> dict:
        """Derived core quantities (core/params.py:201-226)."""
        lsx = p.lsx if p.lsx is not None else p.xsize / (p.xlen - 1)
        lsy = p.lsy if p.lsy is not None else p.ysize / (p.ylen - 1)
        lsz = p.lsz if p.lsz is not None else p.zsize / (p.zlen - 1)
        dim_grid = p.xlen * p.ylen * p.zlen
        return dict(
            xlen=p.xlen, ylen=p.ylen, zlen=p.zlen, halo=p.halo,
            number_coordinates=p.number_coordinates,
            number_total_fields=int(p.number_total_fields),
            dim_grid=dim_grid, dim_fields=int(p.number_total_fields) * dim_grid,
            killkinen=1 if p.killkinen else 0, newtonflow=1 if p.newtonflow else 0,
            unit_length=1 if p.unit_length else 0,
            xsize=float(p.xsize), ysize=float(p.ysize), zsize=float(p.zsize),
            lsx=float(lsx), lsy=float(lsy), lsz=float(lsz),
            grid_volume=float(lsx * lsy * lsz),
            time_step=float(p.time_step if p.time_step is not None else p.courant * lsx),
        )

    @staticmethod
    def from_params(p: Params) -> "ResolvedParams":
        return ResolvedParams(**ResolvedParams.core_values(p))


def default_params(**overrides) -> Params:
    return Params().with_(**overrides)


def pack_device_params(rp: ResolvedParams):
    """(p_i int32[11], p_f float64[8]) in the reference's order (core/params.py:228-267)."""
    p_i = np.array([rp.xlen, rp.ylen, rp.zlen, rp.halo, rp.number_coordinates, rp.number_total_fields,
                    rp.dim_grid, rp.dim_fields, rp.killkinen, rp.newtonflow, rp.unit_length], dtype=np.int32)
    p_f = np.array([rp.xsize, rp.ysize, rp.zsize, rp.lsx, rp.lsy, rp.lsz, rp.grid_volume, rp.time_step],
                   dtype=np.float64)
    return p_i, p_f


def dataclass_values(obj) -> dict:
    return {f.name: getattr(obj, f.name) for f in fields(obj)}
