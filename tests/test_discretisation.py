"""The coded force against the coded energy (oracle only, CPU).

The reference evaluates the force with 4th-order second-derivative and 5x5 mixed
stencils and the energy with 4th-order first-derivative stencils, so the force is
the gradient of the discrete energy only up to O(h^4).  This is why H = E + K of
RK4 dynamics is an audit rather than an invariant.  The test measures the
mismatch of a central difference of the energy along a tangent bump against
<g, u> h^3 at two spacings and checks fourth-order convergence.
"""
import numpy as np
import pytest

from oracle import skyrme_oracle as O


def _mismatch(h, L=40, kappa=1.0):
    from skyrmion_solver_b200 import theories as T
    from skyrmion_solver_b200.initial import exp_profile, hedgehog
    th = T.by_short_name("nuclear")
    p = th.params.default_params(xlen=L, ylen=L, zlen=L, lsx=h, lsy=h, lsz=h, xsize=h * (L - 1),
                                 ysize=h * (L - 1), zsize=h * (L - 1), time_step=0.02, killkinen=True,
                                 newtonflow=True, unit_length=True, kappa=kappa)
    p_i, p_f = th.params.pack_device_params(p.resolved())
    p_i, p_f = np.asarray(p_i, np.int32), np.asarray(p_f, np.float64)
    F = hedgehog((L, L, L), (h, h, h), exp_profile(0.8))
    thd = O.THEORIES["nuclear"]
    x = (np.arange(L) - (L - 1) / 2) * h
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    bump = np.exp(-(X ** 2 + Y ** 2 + Z ** 2) / 0.5)
    rng = np.random.default_rng(1)
    u = np.stack([bump * rng.normal() for _ in range(4)])
    u -= (u * F).sum(0) * F                      # tangent to S^3
    eg, _ = O.gradient(thd, F, p_i, p_f)
    pred = (eg * u).sum() * h ** 3
    eps = 1e-5
    fd = (O.energy_density(thd, F + eps * u, p_i, p_f).sum() -
          O.energy_density(thd, F - eps * u, p_i, p_f).sum()) / (2 * eps)
    return abs(fd - pred) / abs(fd)


def test_force_is_the_energy_gradient_to_fourth_order():
    coarse, fine = _mismatch(0.2), _mismatch(0.1)
    assert coarse > 0.1                   # far from consistent on a coarse lattice
    assert fine < coarse / 8.0            # ... and converging at (close to) fourth order


def _smooth_case(name, L=32, h=0.1):
    import math
    from skyrmion_solver_b200 import theories as T
    from skyrmion_solver_b200.initial import hedgehog
    th = T.by_short_name(name)
    extra = {"rho": dict(mpi=0.586, mrho=3.29, c_alpha=0.2256),
             "coulomb": dict(f_pi=105.9, m_pi=138.0, g=4.010, e=0.302822)}.get(name, {})
    p = th.params.default_params(xlen=L, ylen=L, zlen=L, lsx=h, lsy=h, lsz=h, xsize=h * (L - 1),
                                 ysize=h * (L - 1), zsize=h * (L - 1), time_step=0.01, killkinen=False,
                                 newtonflow=True, unit_length=True, **extra)
    p_i, p_f = th.params.pack_device_params(p.resolved())
    p_i, p_f = np.asarray(p_i, np.int32), np.asarray(p_f, np.float64)
    C = int(p_i[5])
    x = (np.arange(L) - (L - 1) / 2) * h
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    F = np.zeros((C, L, L, L))
    F[:4] = hedgehog((L, L, L), (h, h, h), lambda r: math.pi * np.exp(-(r / 0.7) ** 2))
    for a in range(4, C):
        F[a] = 0.2 * np.exp(-((X - 0.1 * (a - 3)) ** 2 + Y ** 2 + (Z + 0.05 * a) ** 2) / 0.3)
    bump = np.exp(-(X ** 2 + Y ** 2 + Z ** 2) / 0.2)
    return p_i, p_f, F, bump


@pytest.mark.parametrize("name", ["nuclear", "omega", "coulomb", "rho", "berger", "lightly_bound"])
def test_dynamics_potential_generates_the_forces(name):
    """The kernels' force is s_c dPhi/dphi_c for the potential Phi that the energy audit reports:
    along pion directions (tangent to S^3) and along the auxiliary components (sign s_c)."""
    from tests import _dynamics as DY
    p_i, p_f, F, bump = _smooth_case(name)
    thd = O.THEORIES[name]
    eg, _ = O.gradient(thd, F, p_i, p_f)
    h3 = p_f[6]
    C = F.shape[0]
    s = DY.kinetic_signs(name, C)
    rng = np.random.default_rng(11)
    blocks = [range(4)] + ([range(4, C)] if C > 4 else [])
    for comps in blocks:
        u = np.zeros_like(F)
        for a in comps:
            u[a] = bump * rng.normal()
        if 0 in comps:
            u[:4] -= (u[:4] * F[:4]).sum(0) * F[:4]
        eps = 1e-5
        dphi = (DY.potential(name, F + eps * u, p_i, p_f) - DY.potential(name, F - eps * u, p_i, p_f)) / (2 * eps)
        force = float(((eg * s[:, None, None, None]) * u).sum() * h3)
        assert abs(dphi - force) <= 0.03 * abs(force), (name, list(comps), dphi, force)


@pytest.mark.parametrize("name", ["omega", "coulomb"])
def test_dynamics_potential_coupling_sign(name):
    """The pion force's dependence on the auxiliary field is the pion variation of the
    potential's coupling term (the part the coded energy omits), with its sign."""
    from tests import _dynamics as DY
    p_i, p_f, F, bump = _smooth_case(name)
    thd = O.THEORIES[name]
    F0 = F.copy()
    F0[4] = 0.0
    dg = O.gradient(thd, F, p_i, p_f)[0] - O.gradient(thd, F0, p_i, p_f)[0]

    def coupling(Fx):   # Phi(F) - Phi(F with the auxiliary field's own terms only) = the coupling term
        return DY.potential(name, Fx, p_i, p_f) - DY.potential(name, np.concatenate([Fx[:4], 0 * Fx[4:]]), p_i, p_f)

    rng = np.random.default_rng(12)
    for _ in range(2):
        u = np.zeros_like(F)
        for a in range(4):
            u[a] = bump * rng.normal()
        u[:4] -= (u[:4] * F[:4]).sum(0) * F[:4]
        eps = 1e-5
        dc = (coupling(F + eps * u) - coupling(F - eps * u)) / (2 * eps)
        force = float((dg * u).sum() * p_f[6])
        assert abs(dc - force) <= 0.05 * abs(force), (name, dc, force)
