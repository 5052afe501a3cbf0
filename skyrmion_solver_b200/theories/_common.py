"""Helpers shared by the theory packages (parameter resolution, module assembly)."""
from __future__ import annotations

import numpy as np

from ..core.params import ResolvedParams as CoreResolvedParams


def ansatz_flags(ansatz):
    """Parse the initial-ansatz name as the reference does (e.g. th/nuclear_skyrme/params.py:144-150)."""
    ans = (ansatz or "hedgehog").lower().strip()
    hedgehog = ans == "hedgehog"
    rational_map = ans in ("rational_map", "rational map", "rational-map")
    uniform = ans == "uniform"
    if not (hedgehog or rational_map or uniform):
        raise ValueError("Unknown ansatz '{0}'. Valid: hedgehog, rational_map, uniform".format(ansatz))
    return dict(ansatz_hedgehog=hedgehog, ansatz_rational_map=rational_map, ansatz_uniform=uniform)


def core_values(p):
    return CoreResolvedParams.core_values(p)


def pack(rp, core_pack, ints, floats):
    p_i_core, p_f_core = core_pack(rp)
    p_i = np.concatenate((p_i_core, np.array(ints, dtype=np.int32)))
    p_f = np.concatenate((p_f_core, np.array(floats, dtype=np.float64)))
    return p_i, p_f


def ansatz_ints(rp):
    return [1 if rp.ansatz_hedgehog else 0, 1 if rp.ansatz_rational_map else 0, 1 if rp.ansatz_uniform else 0]
