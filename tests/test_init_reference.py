"""The reference's own initial configurations (th/<theory>/initial_config.py).

* The NumPy oracle (oracle/init_oracle.py) against the reference's kernels run
  under Numba's CUDA simulator (tests/golden/init.npz, make_golden_init.py).
* The host side of the product (the lump lists of reference_lumps: seeded
  smorgasbord draws, centres, profile lengths, parameter flags) evaluated with
  the oracle's lump functions against the same goldens.
* The device path (sky_init_lumps through Simulation.initialize) against the
  goldens and, on larger lattices and longer lump lists, against the oracle.

Tolerance: 1e-12 absolute on the unit-length Skyrme components (the device's
fused multiply-adds and CUDA's transcendental functions against the
simulator's NumPy / libm arithmetic); extra components are exactly zero except
omega's field, -c_omega B0, checked to 1e-10 relative.
"""
import ctypes
import json
import os

import numpy as np
import pytest

from oracle import init_oracle as I
from oracle import skyrme_oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "init.npz")
TOL = 1e-12


def _cases():
    if not os.path.exists(GOLD):
        return []
    d = np.load(GOLD)
    return sorted({k.rsplit("/", 1)[0] for k in d.files})


def _case(key):
    d = np.load(GOLD)
    short = key.split("/")[0]
    return (short, d[key + "/p_i"], d[key + "/p_f"], json.loads(str(d[key + "/config"])),
            d[key + "/field"], float(d[key + "/velocity_max"]))


CASES = _cases()


def _check(short, p_i, p_f, got, want):
    C = int(p_i[5])
    got = np.asarray(got, np.float64).reshape(C, -1)
    want = np.asarray(want, np.float64).reshape(C, -1)
    assert np.max(np.abs(got[:4] - want[:4])) <= TOL
    if short == "omega":
        scale = max(float(np.max(np.abs(want[4]))), 1e-300)
        assert np.max(np.abs(got[4] - want[4])) <= 1e-10 * scale
    elif C > 4:
        assert np.array_equal(got[4:], want[4:])


def _omega_seed(p_i, p_f, F):
    dims = tuple(int(v) for v in p_i[:3])
    b = O.baryon_density(O.THEORIES["omega"], F.reshape((int(p_i[5]),) + dims), p_i, p_f)
    return -float(p_f[9]) * np.asarray(b).ravel() / float(p_f[6])


# ---------------------------------------------------------------------------
# CPU
# ---------------------------------------------------------------------------
def test_golden_covers_every_theory_and_mode():
    assert len(CASES) >= 6 * 8 + 9
    for short in ("nuclear", "omega", "coulomb", "rho", "berger", "lightly_bound"):
        assert any(k.startswith(short + "/smorgasbord") for k in CASES)


@pytest.mark.parametrize("key", CASES)
def test_oracle_matches_the_reference(key):
    short, p_i, p_f, cfg, want, vmax = _case(key)
    assert vmax == 0.0                                   # the reference zeroes the velocity
    F = I.initial_field(short, p_i, p_f, cfg)
    if short == "omega" and str(cfg.get("mode", "initial")) != "ground":
        F[4] = _omega_seed(p_i, p_f, F).reshape(F.shape[1:])
    _check(short, p_i, p_f, F, want)


@pytest.mark.parametrize("key", CASES)
def test_lump_lists_match_the_reference(key):
    """The product's host logic, evaluated by the oracle's lump functions."""
    from skyrmion_solver_b200.theories._init_common import reference_lumps
    short, p_i, p_f, cfg, want, _ = _case(key)
    lumps, from_vacuum = reference_lumps(short, p_i, p_f, cfg)
    g, _ = I._grid(p_i, p_f)
    acc = np.zeros((4,) + g.shape[1:])
    acc[0] = 1.0
    for k, L in enumerate(lumps):
        if L[0] == 0.0:
            v = I.hedgehog(g, L[2:5], L[11], L[10])
        else:
            v = I.map_lump(g, L[2:5], L[5:8], L[8:11], L[1], L[11], L[12])
        v = I._normalise(v)
        acc = v if (k == 0 and not from_vacuum) else I._normalise(I._qmul(acc, v))
    C = int(p_i[5])
    F = np.zeros((C,) + g.shape[1:])
    F[:4] = acc
    if short == "omega" and str(cfg.get("mode", "initial")) != "ground":
        F[4] = _omega_seed(p_i, p_f, F).reshape(F.shape[1:])
    _check(short, p_i, p_f, F, want)


def test_reference_and_synthetic_configurations_are_told_apart():
    from skyrmion_solver_b200.theories._init_common import is_reference_config
    assert is_reference_config({}) and is_reference_config({"mode": "rational_map", "baryon_number": 3})
    assert is_reference_config({"mode": "smorgasbord", "seed": 2, "count": 4})
    assert not is_reference_config({"mode": "rational_map", "baryon_number": 4, "scale": 2.0})
    assert not is_reference_config({"mode": "cloud", "count": 3})
    assert not is_reference_config({"mode": "hedgehog", "noise": 1e-3})


def test_init_lumps_rejects_bad_lists():
    from skyrmion_solver_b200 import _lib
    lib = _lib.load()
    pi = np.array([8, 8, 8, 2, 3, 4, 512, 2048, 1, 1, 1, 1, 0, 0], dtype=np.int32)
    pf = np.array([1.4, 1.4, 1.4, 0.2, 0.2, 0.2, 0.008, 0.04, 1.0, 1.0, 1.0, 0.0], dtype=np.float64)
    dummy = ctypes.c_void_p(256)
    good = np.zeros((1, 16))
    good[0, 0], good[0, 1], good[0, 11] = 1.0, 2.0, 1.0
    args = (_lib.i32p(pi), len(pi), _lib.f64p(pf), len(pf))
    for bad_entry in ((0, 2.0), (11, 0.0), (3, np.nan)):
        bad = good.copy()
        bad[0, bad_entry[0]] = bad_entry[1]
        assert lib.sky_init_lumps(*args, 1, _lib.f64p(bad), 0, dummy, None) == 1
    assert lib.sky_init_lumps(*args, -1, _lib.f64p(good), 0, dummy, None) == 1
    assert lib.sky_init_lumps(*args, 1, None, 0, dummy, None) == 1
    assert lib.sky_init_lumps(*args, 1, _lib.f64p(good), 0, None, None) == 1


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
def _simulation(short, p_i, p_f, **over):
    from skyrmion_solver_b200 import theories as T
    from skyrmion_solver_b200.core.simulation import Simulation
    from tests.golden.make_golden import theory_params
    th = T.by_short_name(short)
    sim = Simulation(theory_params(short, th, **over), th)
    assert np.array_equal(sim.p_i_h, p_i) and np.array_equal(sim.p_f_h, p_f)
    return sim


_PARAM_OVERRIDES = {
    "smorgasbord_default": {"baryon_number": 2.0},
    "params_map": {"ansatz": "rational_map", "baryon_number": 4.0, "isospin_rotation": 0.2},
    "params_uniform": {"ansatz": "uniform"},
}


@pytest.mark.gpu
@pytest.mark.parametrize("key", CASES)
def test_device_initialize_matches_the_reference(key):
    import torch
    short, p_i, p_f, cfg, want, _ = _case(key)
    sim = _simulation(short, p_i, p_f, **_PARAM_OVERRIDES.get(key.split("/")[1], {}))
    sim.Velocity.fill_(7.0)
    sim.initialize(dict(cfg))
    torch.cuda.synchronize()
    _check(short, p_i, p_f, sim.Field.cpu().numpy(), want)
    assert float(sim.Velocity.abs().max()) == 0.0


@pytest.mark.gpu
@pytest.mark.parametrize("short,cfg", [
    ("nuclear", {"mode": "rational_map", "baryon_number": 6, "isospin_rotation": 1.1}),
    ("nuclear", {"mode": "smorgasbord", "count": 30, "seed": 11, "lump_baryon": 3, "profile_m0": 0.3}),
    ("coulomb", {"ansatz": "hedgehog", "baryon_number": 3, "isospin_rotation": -0.7}),
    ("rho", {"mode": "smorgasbord", "count": 5, "seed": 4, "lump_baryon": 2}),
    ("berger", {"mode": "rational_map", "baryon_number": 8}),
])
def test_device_lumps_match_the_oracle_on_larger_lattices(short, cfg):
    """Anisotropic 41 x 36 x 30 lattice; 30 lumps take two launches of the composing kernel."""
    import torch
    from skyrmion_solver_b200 import theories as T
    from skyrmion_solver_b200.theories._init_common import build_reference_field
    th = T.by_short_name(short)
    p = th.params.default_params(xlen=41, ylen=36, zlen=30, lsx=0.15, lsy=0.17, lsz=0.2)
    p_i, p_f = th.params.pack_device_params(p.resolved())
    p_i, p_f = np.asarray(p_i, np.int32), np.asarray(p_f, np.float64)
    out = torch.full((int(p_i[7]),), 3.0, dtype=torch.float64, device="cuda")
    build_reference_field(short, p_i, p_f, cfg, out)
    torch.cuda.synchronize()
    want = I.initial_field(short, p_i, p_f, cfg)
    _check(short, p_i, p_f, out.cpu().numpy(), want)


class _CAI:
    """A device buffer known only by its __cuda_array_interface__, as a Numba device array is."""

    def __init__(self, t):
        self._t = t
        self.__cuda_array_interface__ = t.__cuda_array_interface__


@pytest.mark.gpu
@pytest.mark.parametrize("key", ["omega/map_b3", "nuclear/smorgasbord", "rho/default"])
def test_initialize_accepts_foreign_device_arrays(key):
    """The theory's initialize as the reference's own Simulation calls it, with buffers that are
    not torch tensors: the field is written through them."""
    import torch
    from skyrmion_solver_b200 import theories as T
    short, p_i, p_f, cfg, want, _ = _case(key)
    th = T.by_short_name(short)
    C, N = int(p_i[5]), int(p_i[6])
    field = torch.zeros(C * N, dtype=torch.float64, device="cuda")
    vel = torch.full((C * N,), 2.0, dtype=torch.float64, device="cuda")
    temp = torch.full((C * N,), 2.0, dtype=torch.float64, device="cuda")
    th.initial_config.initialize(Velocity=_CAI(vel), Field=_CAI(field), Temp=_CAI(temp), p_i_h=p_i, p_f_h=p_f,
                                 p_i_d=None, p_f_d=None, grid3d=None, block3d=None, config=dict(cfg))
    torch.cuda.synchronize()
    _check(short, p_i, p_f, field.cpu().numpy(), want)
    assert float(vel.abs().max()) == 0.0 and float(temp.abs().max()) == 0.0


def test_lump_list_edge_cases():
    """Host rules of the reference's initialize: Python rounding of the default smorgasbord count,
    an unknown ansatz gives the vacuum, negative baryon numbers keep their sign in the lump (the
    kernel rounds |B|), and the mode name is read case- and space-insensitively."""
    from skyrmion_solver_b200.theories._init_common import reference_lumps
    p_i = np.array([10, 10, 10, 2, 3, 4, 1000, 4000, 1, 1, 1, 1, 0, 0], np.int32)
    p_f = np.array([1.8, 1.8, 1.8, 0.2, 0.2, 0.2, 0.008, 0.04, 1.0, 1.0, 2.5, 0.0])
    lumps, vac = reference_lumps("nuclear", p_i, p_f, {"mode": "smorgasbord"})
    assert vac and len(lumps) == 2                       # round(2.5) == 2 (round half to even)
    lumps, vac = reference_lumps("nuclear", p_i, p_f, {"mode": "smorgasbord", "baryon_number": 3.5})
    assert len(lumps) == 4
    lumps, vac = reference_lumps("nuclear", p_i, p_f, {"ansatz": "torus"})
    assert vac and len(lumps) == 0
    lumps, vac = reference_lumps("nuclear", p_i, p_f, {"mode": " Rational_Map ", "baryon_number": -3})
    assert not vac and lumps[0, 0] == 1.0 and lumps[0, 1] == -3.0
    g, _ = I._grid(p_i, p_f)
    F = I.initial_field("nuclear", p_i, p_f, {"mode": " Rational_Map ", "baryon_number": -3})
    v = I._normalise(I.map_lump(g, lumps[0, 2:5], lumps[0, 5:8], lumps[0, 8:11], lumps[0, 1], lumps[0, 11],
                                lumps[0, 12]))
    assert np.array_equal(F[:4], v)
    # theory profile lengths: omega 0.15 min(size), Coulomb 0.4 min(size) / max(|B|, 1)
    size = np.array([1.8, 2.4, 3.0, 0.2, 0.2, 0.2, 0.008, 0.04, 1.0, 1.0, 2.0, 0.0])
    pi5 = np.array([10, 10, 10, 2, 3, 5, 1000, 5000, 1, 1, 1, 4, 1, 0, 0], np.int32)
    om, _ = reference_lumps("omega", pi5, size, {})
    co, _ = reference_lumps("coulomb", pi5, size, {})
    assert om[0, 11] == max(0.15 * 1.8, 1e-6) and co[0, 11] == max(0.4 * 1.8 / 2.0, 1e-6)
    assert om[0, 0] == 0.0 and co[0, 0] == 0.0           # the parameters' hedgehog flag (p_i[12])
