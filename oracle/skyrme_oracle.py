"""FP64 NumPy oracle for the skyrmion_solver lattice engine.

TEST INFRASTRUCTURE ONLY.  This module is the checker: ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline legs of ``bench.py`` import
it.  The product (``skyrmion_solver_b200``) never imports or calls it.

It restates, vectorised over the lattice, the reference's per-site kernels and
the arrested-Newton/RK4 schedule.  Each function cites the reference file:line
it follows (paths relative to the skyrmion_solver project root).  Arithmetic
order follows the reference expressions where that is cheap, so the oracle
agrees with the reference to ~1e-14 relative; the committed golden vectors in
``tests/golden`` (produced by the reference itself under Numba's CUDA
simulator, see ``tests/golden/make_golden.py``) pin it.

Layout (reference ``core/utils.py:21-48``): a field buffer is FP64 SoA with
flat index ``a*N + x*Ly*Lz + y*Lz + z``; here it is viewed as ``(C, X, Y, Z)``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

TWO_PI2 = 2.0 * math.pi * math.pi
FOUR_PI2 = 4.0 * math.pi * math.pi

# ---------------------------------------------------------------------------
# parameter ABI (core/params.py:227-267; th/*/params.py pack_device_params)
# ---------------------------------------------------------------------------


@dataclass
class Grid:
    X: int
    Y: int
    Z: int
    halo: int
    C: int
    h: tuple
    vol: float
    dt: float
    killkinen: int
    unit_length: int

    @staticmethod
    def from_params(p_i, p_f):
        return Grid(int(p_i[0]), int(p_i[1]), int(p_i[2]), int(p_i[3]), int(p_i[5]),
                    (float(p_f[3]), float(p_f[4]), float(p_f[5])), float(p_f[6]),
                    float(p_f[7]), int(p_i[8]), int(p_i[10]))


# ---------------------------------------------------------------------------
# stencils (core/derivatives.py:18-173)
# ---------------------------------------------------------------------------

def _sl(axis, lo, hi):
    s = [slice(None)] * 3
    s[axis] = slice(lo, hi)
    return tuple(s)


def first_derivative(f, axis, h, halo):
    """core/derivatives.py:54-67: (f-2/12 - 2f-1/3 + 2f+1/3 - f+2/12)/h on halo <= i < L-halo, else 0."""
    L = f.shape[axis]
    out = np.zeros_like(f)
    lo, hi = halo, L - halo
    if hi <= lo:
        return out
    fm2 = f[_sl(axis, lo - 2, hi - 2)]
    fm1 = f[_sl(axis, lo - 1, hi - 1)]
    fp1 = f[_sl(axis, lo + 1, hi + 1)]
    fp2 = f[_sl(axis, lo + 2, hi + 2)]
    out[_sl(axis, lo, hi)] = ((1.0 / 12.0) * fm2 - (2.0 / 3.0) * fm1 + (2.0 / 3.0) * fp1
                              - (1.0 / 12.0) * fp2) / h
    return out


def second_derivative(f, axis, h, halo):
    """core/derivatives.py:106-119: (-f-2/12 + 4f-1/3 - 5f0/2 + 4f+1/3 - f+2/12)/h^2, same mask."""
    L = f.shape[axis]
    out = np.zeros_like(f)
    lo, hi = halo, L - halo
    if hi <= lo:
        return out
    fm2 = f[_sl(axis, lo - 2, hi - 2)]
    fm1 = f[_sl(axis, lo - 1, hi - 1)]
    f0 = f[_sl(axis, lo, hi)]
    fp1 = f[_sl(axis, lo + 1, hi + 1)]
    fp2 = f[_sl(axis, lo + 2, hi + 2)]
    out[_sl(axis, lo, hi)] = (-(1.0 / 12.0) * fm2 + (4.0 / 3.0) * fm1 - (5.0 / 2.0) * f0
                              + (4.0 / 3.0) * fp1 - (1.0 / 12.0) * fp2) / (h * h)
    return out


_MIX_OFF = (-2, -1, 0, 1, 2)
_MIX_C = (1.0, -8.0, 0.0, 8.0, -1.0)


def mixed_derivative(f, ax1, ax2, h1, h2, halo):
    """core/derivatives.py:121-173: 5x5 outer-product stencil / (144 h1 h2).

    Mask is strict on both sides: halo < i < L-halo on both axes (so index
    ``halo`` is zero while index ``L-halo-1`` is not).
    """
    out = np.zeros_like(f)
    L1, L2 = f.shape[ax1], f.shape[ax2]
    lo1, hi1 = halo + 1, L1 - halo
    lo2, hi2 = halo + 1, L2 - halo
    if hi1 <= lo1 or hi2 <= lo2:
        return out
    acc = None
    for i in range(5):
        for j in range(5):
            s = [slice(None)] * 3
            s[ax1] = slice(lo1 + _MIX_OFF[i], hi1 + _MIX_OFF[i])
            s[ax2] = slice(lo2 + _MIX_OFF[j], hi2 + _MIX_OFF[j])
            term = _MIX_C[i] * _MIX_C[j] * f[tuple(s)]
            acc = term if acc is None else acc + term
    s = [slice(None)] * 3
    s[ax1] = slice(lo1, hi1)
    s[ax2] = slice(lo2, hi2)
    out[tuple(s)] = (1.0 / (144.0 * h1 * h2)) * acc
    return out


def derivatives(field, g: Grid, comps=None, second=True):
    """All first (3,C,...) and second (3,3,C,...) derivatives, as the gradient kernel computes them
    (core/integrator.py:37-46)."""
    comps = range(field.shape[0]) if comps is None else comps
    C = field.shape[0]
    D = np.zeros((3,) + field.shape)
    S = np.zeros((3, 3) + field.shape) if second else None
    for a in comps:
        f = field[a]
        for i in range(3):
            D[i, a] = first_derivative(f, i, g.h[i], g.halo)
            if second:
                S[i, i, a] = second_derivative(f, i, g.h[i], g.halo)
        if second:
            for (i, j) in ((1, 0), (2, 0), (2, 1)):
                m = mixed_derivative(f, j, i, g.h[j], g.h[i], g.halo)
                S[i, j, a] = m
                S[j, i, a] = m
    del C
    return D, S


# ---------------------------------------------------------------------------
# small algebra (th/nuclear_skyrme/kernels.py:102-194)
# ---------------------------------------------------------------------------

def det3(a00, a01, a02, a10, a11, a12, a20, a21, a22):
    return (a00 * (a11 * a22 - a12 * a21) - a01 * (a10 * a22 - a12 * a20)
            + a02 * (a10 * a21 - a11 * a20))


def det4_cols(c0, c1, c2, c3):
    """Determinant of the 4x4 matrix whose columns are c0..c3 (each a 4-sequence),
    expanded along the first row (th/nuclear_skyrme/kernels.py:155-194)."""
    m00, m10, m20, m30 = c0
    m01, m11, m21, m31 = c1
    m02, m12, m22, m32 = c2
    m03, m13, m23, m33 = c3
    d0 = det3(m11, m12, m13, m21, m22, m23, m31, m32, m33)
    d1 = det3(m10, m12, m13, m20, m22, m23, m30, m32, m33)
    d2 = det3(m10, m11, m13, m20, m21, m23, m30, m31, m33)
    d3 = det3(m10, m11, m12, m20, m21, m22, m30, m31, m32)
    return m00 * d0 - m01 * d1 + m02 * d2 - m03 * d3


def _eps(i, j, k):
    if i == j or j == k or i == k:
        return 0.0
    return 1.0 if (i, j, k) in ((0, 1, 2), (1, 2, 0), (2, 0, 1)) else -1.0


def _unit(mu, like):
    z = np.zeros_like(like)
    o = np.ones_like(like)
    return tuple(o if a == mu else z for a in range(4))


def project(vec, phi, nsky):
    """project_orthogonal_skyrme_field (th/nuclear_skyrme/kernels.py:236-272)."""
    lm = 0.0
    for a in range(nsky):
        lm = lm + vec[a] * phi[a]
    for a in range(nsky):
        vec[a] = vec[a] - lm * phi[a]


def normalise(field, nsky):
    """compute_norm_skyrme_field (th/nuclear_skyrme/kernels.py:196-234); sites with |phi| = 0 are left."""
    s = 0.0
    for a in range(nsky):
        s = s + field[a] * field[a]
    s = np.sqrt(s)
    nz = s != 0.0
    sd = np.where(nz, s, 1.0)
    for a in range(nsky):
        field[a] = np.where(nz, field[a] / sd, field[a])


# ---------------------------------------------------------------------------
# theory point functions
# ---------------------------------------------------------------------------

def _skyrme_quartic(g, D, S, coef):
    """Quartic Skyrme variation loop shared by nuclear / Coulomb / Berger / lightly-bound
    (th/nuclear_skyrme/kernels.py:1109-1138).  ``coef`` multiplies each (i,j) bracket."""
    norm = [D[i, 0] * D[i, 0] + D[i, 1] * D[i, 1] + D[i, 2] * D[i, 2] + D[i, 3] * D[i, 3]
            for i in range(3)]
    for i in range(3):
        for j in range(3):
            if i == j:
                continue
            dn = 0.0
            dd = 0.0
            dot = 0.0
            for b in range(4):
                dn = dn + 2.0 * D[j, b] * S[i, j, b]
                dd = dd + (S[i, i, b] * D[j, b] + D[i, b] * S[i, j, b])
                dot = dot + D[i, b] * D[j, b]
            for a in range(4):
                br = dn * D[i, a] + norm[j] * S[i, i, a] - dd * D[j, a] - dot * S[i, j, a]
                g[a] = g[a] - (br if coef is None else coef * br)


def _cs_coupling(phi, D, dfield, mu):
    """sum_{ijk} eps_ijk d_i(aux) det[e_mu, phi, d_j phi, d_k phi] (th/omega_skyrme/kernels.py:633-690)."""
    e = _unit(mu, phi[0])
    acc = 0.0
    for i in range(3):
        for j in range(3):
            for k in range(3):
                if i == j or j == k or i == k:
                    continue
                cof = det4_cols(e, (phi[0], phi[1], phi[2], phi[3]),
                                (D[j, 0], D[j, 1], D[j, 2], D[j, 3]),
                                (D[k, 0], D[k, 1], D[k, 2], D[k, 3]))
                acc = acc + _eps(i, j, k) * dfield[i] * cof
    return acc


def baryon_det(phi, D):
    return det4_cols((phi[0], phi[1], phi[2], phi[3]), (D[0, 0], D[0, 1], D[0, 2], D[0, 3]),
                     (D[1, 0], D[1, 1], D[1, 2], D[1, 3]), (D[2, 0], D[2, 1], D[2, 2], D[2, 3]))


def grad_nuclear(phi, D, S, pf, pi):
    """th/nuclear_skyrme/kernels.py:1035-1150."""
    mpi2 = pf[8] * pf[8]
    k2 = pf[9] * pf[9]
    g = [np.zeros_like(phi[0]) for _ in range(4)]
    for a in range(4):
        g[a] = g[a] - (S[0, 0, a] + S[1, 1, a] + S[2, 2, a])
    _skyrme_quartic(g, D, S, k2)
    g[0] = g[0] - mpi2
    project(g, phi, int(pi[5]))
    return np.stack(g)


def grad_omega(phi, D, S, pf, pi):
    """th/omega_skyrme/kernels.py:587-743 (C=5: phi0..3, omega)."""
    mass2 = pf[8] * pf[8]
    c_omega = pf[9]
    dom = (D[0, 4], D[1, 4], D[2, 4])
    g = []
    for mu in range(4):
        gm = np.zeros_like(phi[0])
        e = _unit(mu, phi[0])
        for i in range(3):
            gm = gm - 0.25 * S[i, i, mu]
            for j in range(3):
                for k in range(3):
                    if i == j or j == k or i == k:
                        continue
                    cof = det4_cols(e, (phi[0], phi[1], phi[2], phi[3]),
                                    (D[j, 0], D[j, 1], D[j, 2], D[j, 3]),
                                    (D[k, 0], D[k, 1], D[k, 2], D[k, 3]))
                    gm = gm + c_omega / FOUR_PI2 * _eps(i, j, k) * dom[i] * cof
        if mu == 0:
            gm = gm - 0.25 * mass2
        g.append(gm)
    project(g, phi, int(pi[11]))
    cs = -baryon_det(phi, D) / TWO_PI2
    g_om = phi[4] - (S[0, 0, 4] + S[1, 1, 4] + S[2, 2, 4]) + c_omega * cs
    return np.stack(g + [g_om])


def grad_coulomb(phi, D, S, pf, pi):
    """th/coulomb_skyrme/kernels.py:585-767.  The ``2.0*g`` store at :684-685 is overwritten
    at :751-752, so the pion gradient is the un-doubled g."""
    mass2 = pf[8] * pf[8]
    kappa = pf[9]
    g = [np.zeros_like(phi[0]) for _ in range(4)]
    for a in range(4):
        g[a] = g[a] - (S[0, 0, a] + S[1, 1, a] + S[2, 2, a])
    _skyrme_quartic(g, D, S, None)
    g[0] = g[0] - mass2
    dV = (D[0, 4], D[1, 4], D[2, 4])
    for mu in range(4):
        e = _unit(mu, phi[0])
        for i in range(3):
            for j in range(3):
                for k in range(3):
                    if i == j or j == k or i == k:
                        continue
                    cof = det4_cols(e, (phi[0], phi[1], phi[2], phi[3]),
                                    (D[j, 0], D[j, 1], D[j, 2], D[j, 3]),
                                    (D[k, 0], D[k, 1], D[k, 2], D[k, 3]))
                    g[mu] = g[mu] - kappa / FOUR_PI2 * _eps(i, j, k) * dV[i] * cof
    project(g, phi, int(pi[11]))
    cs = -baryon_det(phi, D) / TWO_PI2
    g_V = 0.0 - (kappa * (S[0, 0, 4] + S[1, 1, 4] + S[2, 2, 4]) + kappa * cs)
    return np.stack(g + [g_V])


def _ridx(i, a):
    """idx_rho (th/rho_skyrme/kernels.py:84-89): rho_i^a at component 4 + 3i + a."""
    return 4 + 3 * i + a


def _dR(S, a, j, k, l):
    return S[j, l, _ridx(k, a)] - S[k, l, _ridx(j, a)]


def _dOmega(D, S, a, j, k, l):
    t = S[j, l, 0] * D[k, a + 1]
    t = t + D[j, 0] * S[k, l, a + 1]
    t = t - S[j, l, a + 1] * D[k, 0]
    t = t - D[j, a + 1] * S[k, l, 0]
    for b in range(3):
        for c in range(3):
            e = _eps(a, b, c)
            if e != 0.0:
                t = t + e * (S[j, l, b + 1] * D[k, c + 1] + D[j, b + 1] * S[k, l, c + 1])
    return t


def _Omega(D, a, i, j):
    t = D[i, 0] * D[j, a + 1] - D[i, a + 1] * D[j, 0]
    for b in range(3):
        for c in range(3):
            e = _eps(a, b, c)
            if e != 0.0:
                t = t + e * D[i, b + 1] * D[j, c + 1]
    return t


def grad_rho(phi, D, S, pf, pi):
    """th/rho_skyrme/kernels.py:597-683 (C=13; c2 = 1, c4 = 1/4)."""
    mpi2 = pf[8] * pf[8]
    mrho2 = pf[9] * pf[9]
    ca = pf[10]
    g = [np.zeros_like(phi[0]) for _ in range(13)]
    for mu in range(4):
        for i in range(3):
            g[mu] = g[mu] - 2.0 * S[i, i, mu]
            for j in range(3):
                for nu in range(4):
                    g[mu] = g[mu] - 2.0 * (
                        S[i, i, mu] * (D[j, nu] * D[j, nu])
                        + (D[i, mu] * (S[i, j, nu] * D[j, nu] - S[j, j, nu] * D[i, nu])
                           - S[i, j, mu] * D[i, nu] * D[j, nu]))
        if mu == 0:
            g[mu] = g[mu] - 2.0 * mpi2
    for a in range(3):
        for i in range(3):
            for j in range(3):
                dR = _dR(S, a, i, j, i)
                g[0] = g[0] + 16.0 * ca * D[j, a + 1] * dR
                g[a + 1] = g[a + 1] - 16.0 * ca * D[j, 0] * dR
                for b in range(3):
                    for c in range(3):
                        e = _eps(b, a, c)
                        if e != 0.0:
                            g[a + 1] = g[a + 1] + 16.0 * ca * e * D[j, c + 1] * _dR(S, b, i, j, i)
    for a in range(3):
        for i in range(3):
            ai = _ridx(i, a)
            val = 8.0 * mrho2 * phi[ai]
            for j in range(3):
                val = val + 8.0 * _dR(S, a, i, j, j)
                val = val - 16.0 * ca * _dOmega(D, S, a, i, j, j)
            g[ai] = val
    project(g, phi, 4)
    return np.stack(g)


def _omega_contract(a, b):
    """th/berger_skyrme/kernels.py:81-111: a0 b3 + a1 b2 - a2 b1 - a3 b0."""
    return a[0] * b[3] + a[1] * b[2] - a[2] * b[1] - a[3] * b[0]


def grad_berger(phi, D, S, pf, pi):
    """th/berger_skyrme/kernels.py:554-736."""
    mpi2 = pf[8] * pf[8]
    k2 = pf[9] * pf[9]
    beta = pf[12] * pf[12] - 1.0
    Fi = [tuple(D[i, a] for a in range(4)) for i in range(3)]
    Sij = {(i, j): tuple(S[i, j, a] for a in range(4)) for i in range(3) for j in range(3)}
    s = tuple(phi[a] for a in range(4))
    g = [np.zeros_like(phi[0]) for _ in range(4)]
    for a in range(4):
        g[a] = g[a] - (S[0, 0, a] + S[1, 1, a] + S[2, 2, a])
    u = [_omega_contract(Fi[i], s) for i in range(3)]
    div_u = _omega_contract(Sij[0, 0], s)
    div_u = div_u + _omega_contract(Sij[1, 1], s)
    div_u = div_u + _omega_contract(Sij[2, 2], s)
    om_phi = (s[3], s[2], -s[1], -s[0])
    om_f = [(Fi[i][3], Fi[i][2], -Fi[i][1], -Fi[i][0]) for i in range(3)]
    for a in range(4):
        g[a] = g[a] - beta * (2.0 * u[0] * om_f[0][a] + 2.0 * u[1] * om_f[1][a]
                              + 2.0 * u[2] * om_f[2][a] + div_u * om_phi[a])
    _skyrme_quartic(g, D, S, k2)
    oc = _omega_contract
    dwxy_dx = oc(Sij[0, 0], Fi[1]) + oc(Fi[0], Sij[0, 1])
    dwxy_dy = oc(Sij[0, 1], Fi[1]) + oc(Fi[0], Sij[1, 1])
    dwxz_dx = oc(Sij[0, 0], Fi[2]) + oc(Fi[0], Sij[0, 2])
    dwxz_dz = oc(Sij[0, 2], Fi[2]) + oc(Fi[0], Sij[2, 2])
    dwyz_dy = oc(Sij[1, 1], Fi[2]) + oc(Fi[1], Sij[1, 2])
    dwyz_dz = oc(Sij[1, 2], Fi[2]) + oc(Fi[1], Sij[2, 2])
    for a in range(4):
        g[a] = g[a] - k2 * beta * (dwxy_dx * om_f[1][a] - dwxy_dy * om_f[0][a]
                                   + dwxz_dx * om_f[2][a] - dwxz_dz * om_f[0][a]
                                   + dwyz_dy * om_f[2][a] - dwyz_dz * om_f[1][a])
    g[0] = g[0] - mpi2
    project(g, phi, int(pi[5]))
    return np.stack(g)


def grad_lightly_bound(phi, D, S, pf, pi):
    """th/lightly_bound_skyrme/kernels.py:567-684."""
    mpi2 = pf[8] * pf[8]
    alpha = pf[9]
    s0 = phi[0]
    g = [np.zeros_like(phi[0]) for _ in range(4)]
    for a in range(4):
        g[a] = g[a] - 2.0 * (1.0 - alpha) * (S[0, 0, a] + S[1, 1, a] + S[2, 2, a])
    _skyrme_quartic(g, D, S, None)
    g[0] = g[0] - (1.0 - alpha) * 2.0 * mpi2
    g[0] = g[0] - 4.0 * alpha * (1.0 - s0) * (1.0 - s0) * (1.0 - s0)
    project(g, phi, int(pi[5]))
    return np.stack(g)


# ---------------------------------------------------------------------------
# energy densities (per site, multiplied by the cell volume)
# ---------------------------------------------------------------------------

def _n_d(D):
    n = [D[i, 0] * D[i, 0] + D[i, 1] * D[i, 1] + D[i, 2] * D[i, 2] + D[i, 3] * D[i, 3]
         for i in range(3)]

    def dot(i, j):
        return D[i, 0] * D[j, 0] + D[i, 1] * D[j, 1] + D[i, 2] * D[j, 2] + D[i, 3] * D[j, 3]
    return n, dot(0, 1), dot(0, 2), dot(1, 2)


def energy_nuclear(phi, D, pf):
    """th/nuclear_skyrme/kernels.py:277-347."""
    (nx, ny, nz), dxy, dxz, dyz = _n_d(D)
    e = 0.5 * (nx + ny + nz)
    e = e + 0.5 * (pf[9] * pf[9]) * ((nx * ny - dxy * dxy) + (nx * nz - dxz * dxz)
                                      + (ny * nz - dyz * dyz))
    e = e + (pf[8] * pf[8]) * (1.0 - phi[0])
    return e * pf[6]


def energy_omega(phi, D, pf):
    """th/omega_skyrme/kernels.py:231-302 (the -c_omega*omega*B0 coupling is not in it, :301)."""
    (nx, ny, nz), _, _, _ = _n_d(D)
    e = 0.125 * (nx + ny + nz)
    e = e + (pf[8] * pf[8]) * 0.25 * (1.0 - phi[0])
    e = e + 0.5 * phi[4] * phi[4]
    e = e + 0.5 * (D[0, 4] * D[0, 4] + D[1, 4] * D[1, 4] + D[2, 4] * D[2, 4])
    return e * pf[6]


def energy_coulomb(phi, D, pf):
    """th/coulomb_skyrme/kernels.py:231-306 (the A0*B0 coupling is not in it, :305)."""
    (nx, ny, nz), dxy, dxz, dyz = _n_d(D)
    e = nx + ny + nz
    e = e + ((nx * ny - dxy * dxy) + (nx * nz - dxz * dxz) + (ny * nz - dyz * dyz))
    e = e + 2.0 * (pf[8] * pf[8]) * (1.0 - phi[0])
    e = e + 0.5 * pf[9] * (D[0, 4] * D[0, 4] + D[1, 4] * D[1, 4] + D[2, 4] * D[2, 4])
    return e * pf[6]


def energy_rho(phi, D, pf):
    """th/rho_skyrme/kernels.py:293-348."""
    mpi2 = pf[8] * pf[8]
    mrho2 = pf[9] * pf[9]
    ca = pf[10]
    e = 0.0
    for i in range(3):
        for mu in range(4):
            e = e + D[i, mu] * D[i, mu]
    for i in range(3):
        for j in range(3):
            for mu in range(4):
                for nu in range(4):
                    e = e + 0.5 * ((D[i, mu] * D[j, nu]) * (D[i, mu] * D[j, nu])
                                   - D[i, mu] * D[j, mu] * D[i, nu] * D[j, nu])
    e = e + 2.0 * mpi2 * (1.0 - phi[0])
    for a in range(3):
        for i in range(3):
            r = phi[_ridx(i, a)]
            e = e + 4.0 * mrho2 * r * r
            for j in range(3):
                Rij = D[i, _ridx(j, a)] - D[j, _ridx(i, a)]
                e = e + 2.0 * Rij * Rij
                e = e - 8.0 * ca * Rij * _Omega(D, a, i, j)
    return e * pf[6]


def energy_berger(phi, D, pf):
    """th/berger_skyrme/kernels.py:251-337."""
    (nx, ny, nz), dxy, dxz, dyz = _n_d(D)
    s = tuple(phi[a] for a in range(4))
    Fi = [tuple(D[i, a] for a in range(4)) for i in range(3)]
    beta = pf[12] * pf[12] - 1.0
    k2 = pf[9] * pf[9]
    ux, uy, uz = (_omega_contract(Fi[i], s) for i in range(3))
    wxy = _omega_contract(Fi[0], Fi[1])
    wxz = _omega_contract(Fi[0], Fi[2])
    wyz = _omega_contract(Fi[1], Fi[2])
    e = 0.5 * (nx + ny + nz)
    e = e + 0.5 * beta * (ux * ux + uy * uy + uz * uz)
    e = e + 0.5 * k2 * ((nx * ny - dxy * dxy) + (nx * nz - dxz * dxz) + (ny * nz - dyz * dyz))
    e = e + 0.5 * k2 * beta * (wxy * wxy + wxz * wxz + wyz * wyz)
    e = e + (pf[8] * pf[8]) * (1.0 - s[0])
    return e * pf[6]


def energy_lightly_bound(phi, D, pf):
    """th/lightly_bound_skyrme/kernels.py:275-346."""
    (nx, ny, nz), dxy, dxz, dyz = _n_d(D)
    alpha = pf[9]
    s0 = phi[0]
    e = (1.0 - alpha) * (nx + ny + nz)
    e = e + 0.5 * ((nx * ny - dxy * dxy) + (nx * nz - dxz * dxz) + (ny * nz - dyz * dyz))
    e = e + (1.0 - alpha) * 2.0 * (pf[8] * pf[8]) * (1.0 - s0)
    e = e + alpha * (1.0 - s0) * (1.0 - s0) * (1.0 - s0) * (1.0 - s0)
    return e * pf[6]


def baryon_density_std(phi, D, pf):
    """th/nuclear_skyrme/kernels.py:385-447: -det[phi, Fx, Fy, Fz] * h^3/(2 pi^2)."""
    return -baryon_det(phi, D) * (pf[6] / TWO_PI2)


def baryon_density_cs(phi, D, pf):
    """th/omega_skyrme/kernels.py:444-500 (also Coulomb): h^3 * (-det/(2 pi^2))."""
    return pf[6] * (-baryon_det(phi, D) / TWO_PI2)


@dataclass(frozen=True)
class TheoryDef:
    name: str
    C: int
    grad: object
    energy: object
    baryon: object
    nsky_index: int | None  # p_i slot holding the number of Skyrme components; None = literal 4
    energy_comps: str = "all"  # derivative components the energy kernel computes


THEORIES = {
    "nuclear": TheoryDef("nuclear", 4, grad_nuclear, energy_nuclear, baryon_density_std, 5),
    "omega": TheoryDef("omega", 5, grad_omega, energy_omega, baryon_density_cs, 11),
    "coulomb": TheoryDef("coulomb", 5, grad_coulomb, energy_coulomb, baryon_density_cs, 11),
    "rho": TheoryDef("rho", 13, grad_rho, energy_rho, baryon_density_std, None),
    "berger": TheoryDef("berger", 4, grad_berger, energy_berger, baryon_density_std, 5),
    "lightly_bound": TheoryDef("lightly_bound", 4, grad_lightly_bound, energy_lightly_bound,
                               baryon_density_std, 5),
}


def nsky(theory: TheoryDef, p_i):
    return 4 if theory.nsky_index is None else int(p_i[theory.nsky_index])


# ---------------------------------------------------------------------------
# kernels as the reference launches them
# ---------------------------------------------------------------------------

def gradient(theory, field, p_i, p_f):
    """_do_gradient_step_kernel (core/integrator.py:37-46) + the theory point fn.
    Returns (EnergyGradient, l = -dt*EG)."""
    g = Grid.from_params(p_i, p_f)
    D, S = derivatives(field, g)
    eg = theory.grad(field, D, S, p_f, p_i)
    return eg, -g.dt * eg


def energy_density(theory, field, p_i, p_f):
    """compute_energy_kernel (e.g. th/nuclear_skyrme/kernels.py:350-382)."""
    g = Grid.from_params(p_i, p_f)
    D, _ = derivatives(field, g, second=False)
    return theory.energy(field, D, p_f)


def baryon_density(theory, field, p_i, p_f):
    """compute_skyrmion_number_kernel (e.g. th/nuclear_skyrme/kernels.py:450-482)."""
    g = Grid.from_params(p_i, p_f)
    D, _ = derivatives(field, g, comps=range(4), second=False)
    return theory.baryon(field, D, p_f)


def block_tree_sum(values):
    """compute_sum (core/utils.py:201-239, 321-346): 1024-wide shared-memory tree per block,
    then numpy's sum of the block partials."""
    v = np.asarray(values, dtype=np.float64).ravel()
    n = v.size
    nb = (n + 1023) // 1024
    buf = np.zeros(nb * 1024)
    buf[:n] = v
    buf = buf.reshape(nb, 1024)
    stride = 512
    while stride > 0:
        buf[:, :stride] = buf[:, :stride] + buf[:, stride:2 * stride]
        stride //= 2
    return float(buf[:, 0].sum())


def arresting_power(velocity, eg):
    """Lattice sum of sum_a V_a EG_a (arresting_criteria, core/integrator.py:178-282), exact
    (math.fsum) on the per-site powers summed in component order."""
    import math as _m
    C = velocity.shape[0]
    v = velocity.reshape(C, -1)
    g = eg.reshape(C, -1)
    site = np.zeros(v.shape[1])
    for a in range(C):
        site = site + v[a] * g[a]
    return site, _m.fsum(site.tolist())


def signed_max(values):
    """compute_max_field (core/utils.py:241-279, 402-424): signed maximum over all entries."""
    return float(np.max(values))


def total_energy(theory, field, p_i, p_f):
    return block_tree_sum(energy_density(theory, field, p_i, p_f))


def total_baryon(theory, field, p_i, p_f):
    return block_tree_sum(baryon_density(theory, field, p_i, p_f))


def _grid_points(p_i, p_f):
    """create_grid_kernel (th/nuclear_skyrme/kernels.py:27-56): r = (h_x i, h_y j, h_z k)."""
    X, Y, Z = (int(v) for v in p_i[:3])
    return np.meshgrid(p_f[3] * np.arange(X), p_f[4] * np.arange(Y), p_f[5] * np.arange(Z), indexing="ij")


def center_of_mass(theory, field, p_i, p_f):
    """compute_center_of_mass (th/nuclear_skyrme/observables.py:182-221 with
    compute_center_of_mass_kernel, kernels.py:678-718): sum b r / sum b; zeros when |B| < 1e-30."""
    b = baryon_density(theory, field, p_i, p_f)
    x, y, z = _grid_points(p_i, p_f)
    B = block_tree_sum(b)
    if abs(B) < 1.0e-30:
        return np.zeros(3)
    return np.array([block_tree_sum(b * x), block_tree_sum(b * y), block_tree_sum(b * z)]) / B


def rms_radius(theory, field, p_i, p_f):
    """compute_rms_radius (th/nuclear_skyrme/observables.py:224-270 with compute_rms_radius_kernel,
    kernels.py:720-758): sqrt(max(sum |r - COM|^2 |b| / sum b, 0)); 0 when |B| < 1e-30."""
    b = baryon_density(theory, field, p_i, p_f)
    B = block_tree_sum(b)
    if abs(B) < 1.0e-30:
        return 0.0
    com = center_of_mass(theory, field, p_i, p_f)
    x, y, z = _grid_points(p_i, p_f)
    num = block_tree_sum(((x - com[0]) ** 2 + (y - com[1]) ** 2 + (z - com[2]) ** 2) * np.abs(b))
    return float(np.sqrt(max(num / B, 0.0)))


# ---------------------------------------------------------------------------
# nuclear-model diagnostics (th/nuclear_skyrme/kernels.py:484-1033,
# observables.py:273-487)
# ---------------------------------------------------------------------------
_EPS3 = np.zeros((3, 3, 3))
for _i, _j, _k in ((0, 1, 2), (1, 2, 0), (2, 0, 1)):
    _EPS3[_i, _j, _k] = 1.0
    _EPS3[_i, _k, _j] = -1.0


def _currents(field, D):
    """_build_left_and_iso_currents (kernels.py:484-547): left currents lcur[k, a] and
    isorotation currents tcur[i, a], arrays of shape (3, 3, X, Y, Z)."""
    s = field[0]
    pi = field[1:4]
    lcur = np.empty((3, 3) + s.shape)
    for k in range(3):
        ds = D[k, 0]
        dp = D[k, 1:4]
        cross = np.stack([pi[1] * dp[2] - pi[2] * dp[1], pi[2] * dp[0] - pi[0] * dp[2],
                          pi[0] * dp[1] - pi[1] * dp[0]])
        for a in range(3):
            lcur[k, a] = s * dp[a] - pi[a] * ds + cross[a]
    pi2 = (pi ** 2).sum(axis=0)
    tcur = np.empty((3, 3) + s.shape)
    for i in range(3):
        for a in range(3):
            v = pi[i] * pi[a] - (pi2 if i == a else 0.0)
            tcur[i, a] = v + s * sum(_EPS3[i, a, b] * pi[b] for b in range(3))
    return lcur, tcur


def _gram(a, b):
    return np.einsum("iaxyz,jaxyz->ijxyz", a, b)


def _site_tensors(field, p_i, p_f):
    g = Grid.from_params(p_i, p_f)
    D, _ = derivatives(field, g, comps=range(4), second=False)
    lcur, tcur = _currents(field, D)
    LL, TT, LT = _gram(lcur, lcur), _gram(tcur, tcur), _gram(tcur, lcur)
    return D, lcur, tcur, LL, TT, LT


def _r_minus_com(theory, field, p_i, p_f):
    com = center_of_mass(theory, field, p_i, p_f)
    x, y, z = _grid_points(p_i, p_f)
    return np.stack([x - com[0], y - com[1], z - com[2]])


def _sum9(t):
    return np.array([[block_tree_sum(t[i, j]) for j in range(3)] for i in range(3)])


def u_tensor(theory, field, p_i, p_f):
    """compute_U_tensor: sum of 2 U0 h^3, U0 = TT + kappa^2 sum_k (TT_ij LL_kk - LT_ik LT_jk)
    (_compute_U0_and_A, kernels.py:548-612; compute_U_tensor_kernel, :813-851)."""
    k2 = p_f[9] * p_f[9]
    _, _, _, LL, TT, LT = _site_tensors(field, p_i, p_f)
    trLL = LL[0, 0] + LL[1, 1] + LL[2, 2]
    U0 = TT + k2 * (TT * trLL - np.einsum("ikxyz,jkxyz->ijxyz", LT, LT))
    return _sum9(2.0 * U0 * p_f[6])


def v_tensor(theory, field, p_i, p_f):
    """compute_V_tensor: sum of 2 h^3 eps_ilm eps_jnp r_l r_n A_mp, A = LL + kappa^2 sum_k
    (LL_ij LL_kk - LL_ik LL_jk), r from the centre of mass (kernels.py:852-905)."""
    k2 = p_f[9] * p_f[9]
    _, _, _, LL, _, _ = _site_tensors(field, p_i, p_f)
    trLL = LL[0, 0] + LL[1, 1] + LL[2, 2]
    A = LL + k2 * (LL * trLL - np.einsum("ikxyz,jkxyz->ijxyz", LL, LL))
    r = _r_minus_com(theory, field, p_i, p_f)
    V = np.einsum("ilm,jnp,lxyz,nxyz,mpxyz->ijxyz", _EPS3, _EPS3, r, r, A)
    return _sum9(2.0 * V * p_f[6])


def w_tensor(theory, field, p_i, p_f):
    """compute_W_tensor: sum of 2 h^3 eps_jlm r_l B_im, B = LT + kappa^2 sum_k (LT_im LL_kk -
    LT_ik LL_mk) (kernels.py:906-975)."""
    k2 = p_f[9] * p_f[9]
    _, _, _, LL, _, LT = _site_tensors(field, p_i, p_f)
    trLL = LL[0, 0] + LL[1, 1] + LL[2, 2]
    Bm = LT + k2 * (LT * trLL - np.einsum("ikxyz,mkxyz->imxyz", LT, LL))
    r = _r_minus_com(theory, field, p_i, p_f)
    W = np.einsum("jlm,lxyz,imxyz->ijxyz", _EPS3, r, Bm)
    return _sum9(2.0 * W * p_f[6])


def quadrupole_tensor(theory, field, p_i, p_f):
    """compute_quadrupole_tensor: sum of (3 r_i r_j - delta_ij r^2) b / 2 (kernels.py:760-812)."""
    b = baryon_density(theory, field, p_i, p_f)
    r = _r_minus_com(theory, field, p_i, p_f)
    r2 = (r ** 2).sum(axis=0)
    Q = 3.0 * np.einsum("ixyz,jxyz->ijxyz", r, r)
    for i in range(3):
        Q[i, i] -= r2
    return _sum9(Q * (0.5 * b))


def d_term(theory, field, p_i, p_f):
    """compute_D_term: -(2/5) E sum h^3 (r_i r_j T_ij - r^2 tr T / 3), T the stress tensor
    (_compute_stress_tensor, kernels.py:614-676; compute_D_integrand_kernel, :976-1033;
    observables.py:440-487)."""
    m2 = p_f[8] * p_f[8]
    k2 = p_f[9] * p_f[9]
    _, _, _, LL, _, _ = _site_tensors(field, p_i, p_f)
    trD = LL[0, 0] + LL[1, 1] + LL[2, 2]
    quartic = sum(LL[i, i] * LL[j, j] - LL[i, j] * LL[i, j] for i in range(3) for j in range(i + 1, 3))
    e = 0.5 * trD + 0.5 * k2 * quartic + m2 * (1.0 - field[0])
    T = LL + k2 * (trD * LL - np.einsum("ikxyz,kjxyz->ijxyz", LL, LL))
    for i in range(3):
        T[i, i] -= e
    r = _r_minus_com(theory, field, p_i, p_f)
    r2 = (r ** 2).sum(axis=0)
    trT = T[0, 0] + T[1, 1] + T[2, 2]
    scalar = np.einsum("ixyz,jxyz,ijxyz->xyz", r, r, T) - r2 * trT / 3.0
    E = total_energy(theory, field, p_i, p_f)
    return -(2.0 / 5.0) * E * block_tree_sum(scalar * p_f[6])


def rk4_stage(V, l_in, F, k_prev, factor, dt):
    """do_rk4_step_kernel (core/integrator.py:50-92): k = dt(V + c l); Temp = F + c k_prev."""
    return dt * (V + factor * l_in), F + factor * k_prev


def rk4_finalize(theory, V, F, ks, ls, p_i):
    """_do_rk4_kernel (core/integrator.py:163-175) + theory norm / projection."""
    k1, k2, k3, k4 = ks
    l1, l2, l3, l4 = ls
    V = V + (1.0 / 6.0) * (l1 + 2.0 * l2 + 2.0 * l3 + l4)
    F = F + (1.0 / 6.0) * (k1 + 2.0 * k2 + 2.0 * k3 + k4)
    if int(p_i[10]):
        ns = nsky(theory, p_i)
        Fl = [F[a] for a in range(F.shape[0])]
        normalise(Fl, ns)
        Vl = [V[a] for a in range(V.shape[0])]
        project(Vl, Fl, ns)
        F = np.stack(Fl)
        V = np.stack(Vl)
    return V, F


def arrested_newton_step(theory, F, V, p_i, p_f, prev_energy, keep_stages=False):
    """do_arrested_newton_flow (core/integrator.py:284-410).

    Returns (F, V, E_new, err, EG_stage4[, stages]).  Intermediate stage fields are not
    renormalised (the reference's normalize_field is a no-op for every theory).
    """
    dt = float(p_f[7])
    k1, T = rk4_stage(V, V, F, F, 0.0, dt)
    eg, l1 = gradient(theory, T, p_i, p_f)
    k2, T = rk4_stage(V, l1, F, k1, 0.5, dt)
    eg, l2 = gradient(theory, T, p_i, p_f)
    k3, T = rk4_stage(V, l2, F, k2, 0.5, dt)
    eg, l3 = gradient(theory, T, p_i, p_f)
    k4, T = rk4_stage(V, l3, F, k3, 1.0, dt)
    eg, l4 = gradient(theory, T, p_i, p_f)
    V, F = rk4_finalize(theory, V, F, (k1, k2, k3, k4), (l1, l2, l3, l4), p_i)
    E = total_energy(theory, F, p_i, p_f)
    if int(p_i[8]) and E > prev_energy:
        V = np.zeros_like(V)
    err = signed_max(eg)
    if keep_stages:
        return F, V, E, err, eg, dict(k1=k1, k2=k2, k3=k3, k4=k4, l1=l1, l2=l2, l3=l3, l4=l4,
                                      Temp=T)
    return F, V, E, err, eg


def potential_density(field, p_i):
    """compute_potential_kernel (th/omega_skyrme/kernels.py:413-441): copies comp p_i[11]."""
    return field[int(p_i[11])].copy()


def rho_meson_density(field):
    """compute_rho_meson_kernel (th/rho_skyrme/kernels.py:385-412): sum_{a>=4} F_a^2 (onto zero)."""
    out = np.zeros_like(field[0])
    for a in range(4, field.shape[0]):
        out = out + field[a] * field[a]
    return out
