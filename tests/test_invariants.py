"""Known-answer invariants of the reference's discretisation, on the oracle (CPU).

The reference ships no tests; besides the golden vectors, these pin properties that any
faithful restatement has:
  * the vacuum phi = (1, 0, 0, 0) (auxiliary fields zero) has zero energy density, zero
    gradient and zero baryon density (up to the rounding of the reference's stencil
    weights, which do not cancel exactly on a constant field: derivatives of ~1e-17);
  * a hedgehog on a large enough lattice has baryon number close to 1;
  * the two-site boundary shell, where every derivative is masked, stays exactly at the
    vacuum under arrested-Newton steps.
"""
import numpy as np
import pytest

from oracle import skyrme_oracle as O

NAMES = ["nuclear", "omega", "coulomb", "rho", "berger", "lightly_bound"]
EXTRA = {"rho": dict(mpi=0.586, mrho=3.29, c_alpha=0.2256),
         "coulomb": dict(f_pi=105.9, m_pi=138.0, g=4.010, e=0.302822)}


def _params(name, L, h):
    from skyrmion_solver_b200 import theories as T
    th = T.by_short_name(name)
    p = th.params.default_params(xlen=L, ylen=L, zlen=L, lsx=h, lsy=h, lsz=h, xsize=h * (L - 1),
                                 ysize=h * (L - 1), zsize=h * (L - 1), time_step=0.02, killkinen=True,
                                 newtonflow=True, unit_length=True, **EXTRA.get(name, {}))
    p_i, p_f = th.params.pack_device_params(p.resolved())
    return np.asarray(p_i, np.int32), np.asarray(p_f, np.float64)


@pytest.mark.parametrize("name", NAMES)
def test_vacuum_is_a_zero(name):
    p_i, p_f = _params(name, 12, 0.2)
    F = np.zeros((int(p_i[5]), 12, 12, 12))
    F[0] = 1.0
    thd = O.THEORIES[name]
    assert np.max(np.abs(O.energy_density(thd, F, p_i, p_f))) <= 1e-30
    assert np.max(np.abs(O.baryon_density(thd, F, p_i, p_f))) <= 1e-30
    eg, _ = O.gradient(thd, F, p_i, p_f)
    assert np.max(np.abs(eg)) <= 1e-12


@pytest.mark.parametrize("name", ["nuclear", "omega", "berger"])
def test_hedgehog_has_unit_baryon_number(name):
    from skyrmion_solver_b200.initial import exp_profile, hedgehog, with_extra_components
    L, h = 48, 0.15
    p_i, p_f = _params(name, L, h)
    F = with_extra_components(hedgehog((L, L, L), (h, h, h), exp_profile(0.8)), int(p_i[5]))
    B = O.total_baryon(O.THEORIES[name], F, p_i, p_f)
    assert abs(B - 1.0) <= 2e-2, B


@pytest.mark.parametrize("name", ["nuclear", "coulomb", "rho"])
def test_boundary_shell_stays_at_the_vacuum(name):
    from skyrmion_solver_b200.initial import exp_profile, hedgehog, vacuum_shell, with_extra_components
    L, h = 20, 0.2
    p_i, p_f = _params(name, L, h)
    F = with_extra_components(hedgehog((L, L, L), (h, h, h), exp_profile(1.0)), int(p_i[5]))
    vacuum_shell(F, 2)
    V = np.zeros_like(F)
    thd = O.THEORIES[name]
    E = O.total_energy(thd, F, p_i, p_f)
    for _ in range(2):
        F, V, E, err, _ = O.arrested_newton_step(thd, F, V, p_i, p_f, E)
    shell = np.ones((L, L, L), bool)
    shell[2:-2, 2:-2, 2:-2] = False
    assert np.all(F[0][shell] == 1.0)
    assert np.all(F[1:][:, shell] == 0.0)


def test_centre_of_mass_and_radius_of_a_displaced_hedgehog():
    """The oracle's centre of mass (reference grid r = h * index) sits at the hedgehog's centre;
    a symmetric hedgehog's RMS radius does not depend on where it sits."""
    from skyrmion_solver_b200.initial import exp_profile, hedgehog
    L, h = 40, 0.2
    p_i, p_f = _params("nuclear", L, h)
    thd = O.THEORIES["nuclear"]
    mid = (L - 1) / 2.0 * h
    r0 = []
    for c in ((0.0, 0.0, 0.0), (0.4, -0.2, 0.2)):
        F = hedgehog((L, L, L), (h, h, h), exp_profile(0.7), center=c)
        com = O.center_of_mass(thd, F, p_i, p_f)
        assert np.max(np.abs(com - (mid + np.asarray(c)))) <= 2e-3, com
        r0.append(O.rms_radius(thd, F, p_i, p_f))
    assert abs(r0[0] - r0[1]) <= 1e-2 * r0[0]
