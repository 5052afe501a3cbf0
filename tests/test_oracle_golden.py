"""The CPU oracle against the reference's own outputs (golden vectors produced by the
reference kernels under Numba's CUDA simulator).  The oracle reproduces them
bit for bit; the bound below allows 1e-13 relative in case numpy changes its
summation order."""
import numpy as np
import pytest

from oracle import skyrme_oracle as O
from tests import _golden as G

TOL = 1e-13


@pytest.fixture(params=G.available())
def gold(request):
    return request.param, G.load(request.param)


def test_gradient_kernel(gold):
    name, d = gold
    eg, l = O.gradient(O.THEORIES[name], d["temp_in"], d["p_i"], d["p_f"])
    assert G.rel_err(eg, d["grad_eg"]) <= TOL
    assert G.rel_err(l, d["grad_l"]) <= TOL


def test_densities_and_totals(gold):
    name, d = gold
    th = O.THEORIES[name]
    F = d["field0"]
    assert G.rel_err(O.energy_density(th, F, d["p_i"], d["p_f"]), d["energy_density0"]) <= TOL
    assert G.rel_err(O.baryon_density(th, F, d["p_i"], d["p_f"]), d["baryon_density0"]) <= TOL
    assert abs(O.total_energy(th, F, d["p_i"], d["p_f"]) - d["energy0"]) <= TOL * abs(d["energy0"])
    assert abs(O.total_baryon(th, F, d["p_i"], d["p_f"]) - d["baryon0"]) <= 1e-12
    if "potential_density0" in d:
        assert G.rel_err(O.potential_density(F, d["p_i"]), d["potential_density0"]) == 0.0
    if "rho_meson_density0" in d:
        assert G.rel_err(O.rho_meson_density(F), d["rho_meson_density0"]) <= TOL


def test_arrested_newton_steps(gold):
    name, d = gold
    th = O.THEORIES[name]
    F, V = d["field0"], d["velocity0"]
    nsteps = len(d["energies"])
    for s in range(nsteps):
        F, V, E, err, eg, *st = O.arrested_newton_step(th, F, V, d["p_i"], d["p_f"], float(d[f"prev{s}"]),
                                                       keep_stages=(s == 0))
        assert G.rel_err(F, d[f"field{s + 1}"]) <= TOL
        assert G.rel_err(eg, d[f"eg{s + 1}"]) <= TOL
        if np.any(d[f"velocity{s + 1}"]):
            assert G.rel_err(V, d[f"velocity{s + 1}"]) <= TOL
        else:  # arrested: the reference zeroed the velocity
            assert not np.any(V)
        assert abs(E - d["energies"][s]) <= TOL * abs(d["energies"][s])
        assert abs(err - d["errs"][s]) <= TOL * abs(d["errs"][s])
        if s == 0:
            for k, v in st[0].items():
                assert G.rel_err(v, d[f"{k}_1"]) <= TOL, k


def test_golden_covers_both_arrest_branches():
    """Step 2 of every fixture is forced to arrest (prev = -1e300), step 1 is not (prev = +1e300)."""
    for name in G.available():
        d = G.load(name)
        assert np.any(d["velocity1"]) and not np.any(d["velocity2"])
