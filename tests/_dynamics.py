"""The potential that the RK4 dynamics of each variant conserves, restated from the oracle.

The kernels integrate phi_c'' = -g_c.  H = (1/2) h^3 sum_c s_c |phi_c'|^2 + Phi is
conserved when g_c = s_c dPhi/dphi_c.  For nuclear, rho, Berger and lightly-bound, Phi
is the coded energy and s_c = 1.  For omega and Coulomb the auxiliary field
(component 4) is the time component of a vector field, with s_4 = -1:
  omega:   Phi = E_pion - E_omega - c_omega * sum(omega B0) h^3
  Coulomb: Phi = E_pion / 2 - (kappa / 2) sum |grad A0|^2 h^3 + kappa * sum(A0 B0) h^3
The signs and factors are what the central-difference checks in
tests/test_discretisation.py establish against the oracle's forces.
"""
import numpy as np

from oracle import skyrme_oracle as O


def _parts(name, F, p_i, p_f):
    thd = O.THEORIES[name]
    g = O.Grid.from_params(p_i, p_f)
    D, _ = O.derivatives(F, g, second=False)
    e = O.energy_density(thd, F, p_i, p_f)           # includes h^3
    vol = p_f[6]
    b0 = -O.baryon_det(F, D) / O.TWO_PI2             # per unit volume
    return D, e, vol, b0


def potential(name, F, p_i, p_f):
    if name not in ("omega", "coulomb"):
        return float(O.energy_density(O.THEORIES[name], F, p_i, p_f).sum())
    D, e, vol, b0 = _parts(name, F, p_i, p_f)
    grad2 = D[0, 4] ** 2 + D[1, 4] ** 2 + D[2, 4] ** 2
    c = p_f[9]
    if name == "omega":
        ew = vol * (0.5 * F[4] ** 2 + 0.5 * grad2)
        dens = (e - ew) - ew - c * F[4] * b0 * vol
    else:
        ev = vol * 0.5 * c * grad2
        dens = 0.5 * (e - ev) - ev + c * F[4] * b0 * vol
    return float(dens.sum())


def kinetic_signs(name, C):
    s = np.ones(C)
    if name in ("omega", "coulomb"):
        s[4] = -1.0
    return s


def kinetic(name, V, p_f):
    s = kinetic_signs(name, V.shape[0])
    return float(0.5 * p_f[6] * (s[:, None, None, None] * V * V).sum())
