"""Nuclear-model diagnostics: the oracle against the reference's own values
(tests/golden/nuclear_diag.npz, produced by make_golden_diag.py under the Numba
CUDA simulator), and the fused device pass against the oracle."""
import os

import numpy as np
import pytest

from oracle import skyrme_oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
DIAG = os.path.join(HERE, "golden", "nuclear_diag.npz")
TOL = 1e-10


def _gold():
    if not os.path.exists(DIAG):
        pytest.skip("nuclear_diag.npz not generated")
    return dict(np.load(DIAG))


def _close(a, b, tol=TOL):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return np.max(np.abs(a - b)) <= tol * max(1.0, float(np.max(np.abs(b))))


def test_oracle_matches_the_reference_diagnostics():
    d = _gold()
    th = O.THEORIES["nuclear"]
    F, p_i, p_f = d["field"], d["p_i"], d["p_f"]
    assert _close(O.center_of_mass(th, F, p_i, p_f), d["com"])
    assert _close(O.rms_radius(th, F, p_i, p_f), d["rms"])
    assert _close(O.u_tensor(th, F, p_i, p_f), d["U"])
    assert _close(O.v_tensor(th, F, p_i, p_f), d["V"])
    assert _close(O.w_tensor(th, F, p_i, p_f), d["W"])
    assert _close(O.quadrupole_tensor(th, F, p_i, p_f), d["Q"])
    assert _close(O.d_term(th, F, p_i, p_f), d["D"])


@pytest.mark.gpu
def test_device_diagnostics_match_the_oracle():
    import torch
    from tests import _golden as G
    from tests._gpu import golden_simulation, host
    d = G.load("nuclear")
    th, sim = golden_simulation("nuclear", d)
    thd = O.THEORIES["nuclear"]
    F, p_i, p_f = d["field0"], d["p_i"], d["p_f"]
    assert _close(sim.compute_U_tensor(), O.u_tensor(thd, F, p_i, p_f))
    assert _close(sim.compute_V_tensor(), O.v_tensor(thd, F, p_i, p_f))
    assert _close(sim.compute_W_tensor(), O.w_tensor(thd, F, p_i, p_f))
    assert _close(sim.compute_quadrupole_tensor(), O.quadrupole_tensor(thd, F, p_i, p_f))
    assert _close(sim.compute_D_term(), O.d_term(thd, F, p_i, p_f))
    torch.cuda.synchronize()
    assert _close(host(sim.com_d), O.center_of_mass(thd, F, p_i, p_f))
    assert not sim.en.any() and not sim.entmp.any()


@pytest.mark.gpu
def test_engine_diagnostics_of_a_resident_instance():
    """Engine.diagnostics on a resident FP64 instance of the golden field gives the reference's
    own values; on a defect-corrected FP32 instance it matches the oracle on the instance's field."""
    import torch
    from skyrmion_solver_b200.engine import Engine
    d = _gold()
    F, p_i, p_f = d["field"], d["p_i"], d["p_f"]
    th = O.THEORIES["nuclear"]
    with Engine(0) as eng:
        i = eng.add("nuclear", (p_i, p_f), F, None, precision="fp64")
        g = eng.diagnostics(i)
        assert _close(g["center_of_mass"], d["com"]) and _close(g["rms_radius"], d["rms"])
        for k, ref in (("U", "U"), ("V", "V"), ("W", "W"), ("quadrupole", "Q"), ("D_term", "D")):
            assert _close(g[k], d[ref]), k
        j = eng.add("nuclear", (p_i, p_f), F, None, precision="fp32d")
        eng.step(3)
        g = eng.diagnostics(j)
        field, _ = eng.view(j)
        torch.cuda.synchronize()
        Fj = field.cpu().numpy().reshape(F.shape)
        assert _close(g["center_of_mass"], O.center_of_mass(th, Fj, p_i, p_f))
        assert _close(g["U"], O.u_tensor(th, Fj, p_i, p_f))
        assert _close(g["D_term"], O.d_term(th, Fj, p_i, p_f))
