"""Parameter packing: this package's p_i / p_f equal the reference's for the same inputs."""
import numpy as np
import pytest

from skyrmion_solver_b200 import theories as T
from tests import _golden as G
from tests.golden.make_golden import theory_params

PKG = {"nuclear": "nuclear_skyrme", "omega": "omega_skyrme", "coulomb": "coulomb_skyrme", "rho": "rho_skyrme",
       "berger": "berger_skyrme", "lightly_bound": "lightly_bound_skyrme"}


@pytest.mark.parametrize("name", G.available())
def test_pack_matches_reference(name):
    d = G.load(name)
    th = T.by_short_name(name)
    p_i, p_f = th.params.pack_device_params(theory_params(name, th).resolved())
    np.testing.assert_array_equal(p_i, d["p_i"])
    np.testing.assert_array_equal(p_f, d["p_f"])


def test_defaults_and_derivations():
    om = T.by_short_name("omega").params.default_params().resolved()
    assert om.mass == pytest.approx(138.0 / 782.0) and om.c_omega == pytest.approx(782.0 * 8.253 / 186.0)
    co = T.by_short_name("coulomb").params.default_params().resolved()
    assert co.mass == pytest.approx(2 * 138.0 / (4.0 * 105.9)) and co.kappa == pytest.approx(16 * 0.302822 ** 2 / 2)
    rho = T.by_short_name("rho").params.default_params(e_skyrme=3.65, f_pi=129.0).resolved()
    assert rho.mpi == pytest.approx(2 * 138.0 / (3.65 * 129.0))
    core = T.by_short_name("nuclear").params.default_params(xlen=64, xsize=12.6, courant=0.5).resolved()
    assert core.lsx == pytest.approx(0.2) and core.time_step == pytest.approx(0.1)


def test_reference_errors():
    with pytest.raises(ValueError):
        T.by_short_name("nuclear").params.default_params(ansatz="bogus").resolved()
    with pytest.raises(ValueError):
        T.by_short_name("omega").params.default_params(m_omega=0.0).resolved()
    with pytest.raises(ValueError):
        T.by_short_name("coulomb").params.default_params(g=0.0).resolved()
    with pytest.raises(KeyError):
        T.load_theory("no such theory")


def test_registry_names():
    names = T.list()
    assert "Nuclear Skyrme model" in names and "Omega-Skyrme model" in names and len(names) == 6
    assert T.load_theory("skyrmions").THEORY_SPEC.name == "Nuclear Skyrme model"
