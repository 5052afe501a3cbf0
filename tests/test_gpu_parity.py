"""Parity of the sm_100a FP64 path (called through the C ABI) with the reference's outputs.

Golden vectors come from the reference kernels themselves (tests/golden); the
tolerances are relative to the largest magnitude of the compared array.  The
FP64 kernels use fused multiply-adds and a different (separable-free,
tile-staged) evaluation order, so they agree to ~1e-14 per kernel and ~1e-12
after three RK4 steps; the stated bound for the energy is 1e-10 relative per step.
"""
import numpy as np
import pytest

from skyrmion_solver_b200.core.launch import DeviceParams
from tests import _golden as G
from tests._gpu import dev, golden_simulation, host

pytestmark = pytest.mark.gpu

KERNEL_TOL = 1e-12
STEP_TOL = 1e-10
ENERGY_TOL = 1e-10


@pytest.fixture(params=G.available())
def gold(request):
    return request.param, G.load(request.param)


def test_gradient_kernel(gold):
    import torch
    name, d = gold
    th, sim = golden_simulation(name, d)
    shp = d["grad_eg"].shape
    T_in = dev(d["temp_in"])
    eg = torch.zeros_like(T_in)
    l = torch.zeros_like(T_in)
    th.kernels.do_gradient_step_kernel[(1, 1, 1), (8, 8, 4)](l, T_in, None, None, eg, sim.p_i_d, sim.p_f_d)
    torch.cuda.synchronize()
    assert G.rel_err(host(eg, shp), d["grad_eg"]) <= KERNEL_TOL
    assert G.rel_err(host(l, shp), d["grad_l"]) <= KERNEL_TOL


def test_gradient_accepts_raw_device_params(gold):
    """p_i / p_f given as plain device tensors (as the reference passes Numba arrays)."""
    import torch
    name, d = gold
    th, sim = golden_simulation(name, d)
    T_in = dev(d["temp_in"])
    eg = torch.zeros_like(T_in)
    l = torch.zeros_like(T_in)
    p_i = torch.from_numpy(d["p_i"]).cuda()
    p_f = torch.from_numpy(d["p_f"]).cuda()
    th.kernels.do_gradient_step_kernel[(1, 1, 1), (8, 8, 4)](l, T_in, None, None, eg, p_i, p_f)
    torch.cuda.synchronize()
    assert G.rel_err(host(eg, d["grad_eg"].shape), d["grad_eg"]) <= KERNEL_TOL


def test_densities(gold):
    import torch
    name, d = gold
    th, sim = golden_simulation(name, d)
    dims = d["energy_density0"].shape
    sim.compute_energy_density()
    assert G.rel_err(host(sim.en, dims), d["energy_density0"]) <= KERNEL_TOL
    sim.compute_baryon_density()
    assert G.rel_err(host(sim.en, dims), d["baryon_density0"]) <= KERNEL_TOL
    if "potential_density0" in d:
        sim.compute_potential_density()
        assert np.array_equal(host(sim.en, dims), d["potential_density0"])
    if "rho_meson_density0" in d:
        sim.en.zero_()
        sim.compute_rho_meson_density()
        assert G.rel_err(host(sim.en, dims), d["rho_meson_density0"]) <= KERNEL_TOL
    torch.cuda.synchronize()


def test_observables(gold):
    name, d = gold
    th, sim = golden_simulation(name, d)
    obs = sim.observables()
    assert abs(obs["energy"] - d["energy0"]) <= ENERGY_TOL * abs(d["energy0"])
    assert abs(obs["skyrmion_number"] - d["baryon0"]) <= 1e-12
    # the reference leaves en / entmp zeroed
    assert not sim.en.any() and not sim.entmp.any()


def test_center_of_mass_and_rms_radius(gold):
    """Simulation.compute_center_of_mass / compute_rms_radius (one fused moments pass) against the
    oracle's restatement of the reference's two kernels and host sums."""
    from oracle import skyrme_oracle as O
    name, d = gold
    th, sim = golden_simulation(name, d)
    thd = O.THEORIES[name]
    com = sim.compute_center_of_mass()
    ref = O.center_of_mass(thd, d["field0"], d["p_i"], d["p_f"])
    assert np.max(np.abs(com - ref)) <= 1e-12 * max(1.0, float(np.max(np.abs(ref))))
    r = sim.compute_rms_radius()
    rref = O.rms_radius(thd, d["field0"], d["p_i"], d["p_f"])
    assert abs(r - rref) <= 1e-10 * max(1.0, abs(rref))
    assert np.allclose(host(sim.com_d), ref, rtol=0, atol=1e-12 * max(1.0, float(np.max(np.abs(ref)))))
    assert not sim.en.any() and not sim.entmp.any()


def test_arrested_newton_steps(gold):
    name, d = gold
    th, sim = golden_simulation(name, d)
    shp = d["field0"].shape
    for s in range(len(d["energies"])):
        E, err = sim.step(float(d[f"prev{s}"]))
        assert abs(E - d["energies"][s]) <= ENERGY_TOL * abs(d["energies"][s]), (s, E, d["energies"][s])
        assert abs(err - d["errs"][s]) <= STEP_TOL * abs(d["errs"][s])
        assert G.rel_err(host(sim.Field, shp), d[f"field{s + 1}"]) <= STEP_TOL
        assert G.rel_err(host(sim.EnergyGradient, shp), d[f"eg{s + 1}"]) <= STEP_TOL
        v = host(sim.Velocity, shp)
        if np.any(d[f"velocity{s + 1}"]):
            assert G.rel_err(v, d[f"velocity{s + 1}"]) <= STEP_TOL
        else:
            assert not np.any(v)
        if s == 0:
            for k in ("k1", "k2", "k3", "k4", "l1", "l2", "l3", "l4", "Temp"):
                assert G.rel_err(host(getattr(sim, k), shp), d[f"{k}_1"]) <= STEP_TOL, k


class _Opaque:
    """Wraps a launchable so the integrator cannot recognise it (forces the unfused schedule)."""

    def __init__(self, k):
        self.k = k

    def __getitem__(self, cfg):
        return self.k[cfg]

    def __call__(self, *a, **kw):
        return self.k(*a, **kw)


def test_unfused_schedule_matches_fused(gold):
    """The Python-driven schedule with individual launches equals the one-call C step."""
    from skyrmion_solver_b200.core.integrator import do_arrested_newton_flow
    name, d = gold
    th, sim_a = golden_simulation(name, d)
    _, sim_b = golden_simulation(name, d)
    for s in range(2):
        prev = float(d[f"prev{s}"])
        ea, erra = sim_a.step(prev)
        eb, errb = do_arrested_newton_flow(
            sim_b.Velocity, sim_b.Field, None, None, sim_b.EnergyGradient, sim_b.k1, sim_b.k2, sim_b.k3, sim_b.k4,
            sim_b.l1, sim_b.l2, sim_b.l3, sim_b.l4, sim_b.Temp, sim_b.en, sim_b.entmp, sim_b.gridsum_partial,
            sim_b.max_partial, sim_b.p_i_d, sim_b.p_f_d, sim_b.p_i_h, sim_b.p_f_h, prev,
            _Opaque(th.observables.compute_energy), _Opaque(th.kernels.do_gradient_step_kernel),
            _Opaque(th.kernels.do_rk4_kernel))
        assert ea == eb and erra == errb
        assert bool((sim_a.Field == sim_b.Field).all()) and bool((sim_a.Velocity == sim_b.Velocity).all())


def test_reductions_exact_and_deterministic():
    import math
    import torch
    from skyrmion_solver_b200.core.utils import compute_max, compute_min, compute_sum
    rng = np.random.default_rng(7)
    for n in (1, 1023, 1024, 1025, 262144, 3_000_001):
        x = rng.standard_normal(n) * 10.0 ** rng.uniform(-8, 8, size=n)
        t = dev(x)
        s1 = compute_sum(t, None, n)
        s2 = compute_sum(t, None, n)
        assert s1 == s2
        assert abs(s1 - math.fsum(x)) <= 1e-15 * np.abs(x).sum() + 1e-300
        assert compute_max(t, None, n) == float(np.max(x))
        assert compute_min(t, None, n) == float(np.min(x))
    assert compute_min(dev(np.arange(3.0, 5000.0)), None, 4997) == 3.0    # all positive: not the padding
    torch.cuda.synchronize()


@pytest.mark.parametrize("name", ["nuclear", "rho"])
def test_arresting_criteria_matches_the_oracle(name):
    """Power V . EG (arresting_criteria, core/integrator.py:178-282) on the golden velocity and
    gradient: the lattice sum to the exact sum's rounding, the per-site values to FMA rounding."""
    import torch
    from oracle import skyrme_oracle as O
    from skyrmion_solver_b200.core.integrator import arresting_criteria, arresting_criteria_kernel
    d = G.load(name)
    V, EG = d["velocity0"], d["grad_eg"]
    site, total = O.arresting_power(V, EG)
    en = torch.full((site.size,), 5.0, dtype=torch.float64, device="cuda")
    entmp = torch.full_like(en, 5.0)
    got = arresting_criteria(dev(V), dev(EG), en, entmp, None, None, d["p_i"])
    assert abs(got - total) <= 1e-15 * np.abs(site).sum()
    assert float(en.abs().max()) == 0.0 and float(entmp.abs().max()) == 0.0
    arresting_criteria_kernel[(1, 1, 1), (8, 8, 4)](dev(V), dev(EG), en, d["p_i"])
    torch.cuda.synchronize()
    assert np.max(np.abs(en.cpu().numpy() - site)) <= 1e-14 * np.abs(site).max()


def test_signed_max_padding_semantics():
    """All-negative input: the signed max is the largest (least negative) entry, not 0."""
    from skyrmion_solver_b200.core.utils import compute_max
    x = -np.arange(1, 5000, dtype=np.float64)
    assert compute_max(dev(x), None, x.size) == -1.0


def test_simulation_initialize_modes():
    import torch
    from skyrmion_solver_b200 import theories as T
    from skyrmion_solver_b200.core.simulation import Simulation
    th = T.load_theory("Nuclear Skyrme model")
    p = th.params.default_params(xlen=24, ylen=24, zlen=24, lsx=0.2, lsy=0.2, lsz=0.2)
    sim = Simulation(p, th)
    sim.initialize({"mode": "ground"})
    assert sim.observables()["energy"] == 0.0
    sim.initialize({"mode": "hedgehog", "scale": 1.0})
    obs = sim.observables()
    assert 0.5 < obs["skyrmion_number"] < 1.05
    g = sim.grid.view(3, -1)
    assert float(g[0, -1]) == pytest.approx(0.2 * 23)
    torch.cuda.synchronize()


class _Foreign:
    """A device array as Numba hands it over: __cuda_array_interface__ plus copy_to_host, and
    slice assignment of a scalar; no torch methods."""

    def __init__(self, t):
        self._t = t
        self.__cuda_array_interface__ = t.__cuda_array_interface__

    def copy_to_host(self):
        return self._t.cpu().numpy()

    def __setitem__(self, key, value):
        self._t[key] = value


@pytest.mark.parametrize("opaque", [False, True])
def test_reference_driver_with_foreign_buffers(gold, opaque):
    """The reference's Simulation.step / observables call pattern with Numba-like buffers: the
    fused call and the per-launch schedule give the same bits as the torch-buffer driver."""
    from skyrmion_solver_b200.core.integrator import do_arrested_newton_flow
    name, d = gold
    th, sim_a = golden_simulation(name, d)
    _, sim_b = golden_simulation(name, d)
    F = {k: _Foreign(getattr(sim_b, k)) for k in ("Velocity", "Field", "EnergyGradient", "k1", "k2", "k3", "k4", "l1",
                                                   "l2", "l3", "l4", "Temp", "en", "entmp", "gridsum_partial",
                                                   "max_partial")}
    p_i_d, p_f_d = _Foreign(sim_b.p_i_d.device), _Foreign(sim_b.p_f_d.device)
    wrap = _Opaque if opaque else (lambda k: k)
    for s in range(2):
        prev = float(d[f"prev{s}"])
        ea, erra = sim_a.step(prev)
        eb, errb = do_arrested_newton_flow(
            F["Velocity"], F["Field"], None, None, F["EnergyGradient"], F["k1"], F["k2"], F["k3"], F["k4"], F["l1"],
            F["l2"], F["l3"], F["l4"], F["Temp"], F["en"], F["entmp"], F["gridsum_partial"], F["max_partial"],
            p_i_d, p_f_d, sim_b.p_i_h, sim_b.p_f_h, prev, wrap(th.observables.compute_energy),
            wrap(th.kernels.do_gradient_step_kernel), wrap(th.kernels.do_rk4_kernel))
        assert ea == eb and erra == errb
        assert bool((sim_a.Field == sim_b.Field).all()) and bool((sim_a.Velocity == sim_b.Velocity).all())
    e = th.observables.compute_energy(F["Field"], None, F["en"], F["entmp"], F["gridsum_partial"], p_i_d, p_f_d,
                                      sim_b.p_i_h, sim_b.p_f_h)
    assert e == sim_a.observables()["energy"]
    assert not sim_b.en.any() and not sim_b.entmp.any()
