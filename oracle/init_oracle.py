"""NumPy oracle for the reference's initial configurations.

TEST INFRASTRUCTURE ONLY.  ``tests/`` imports this module as the checker; the
product (``skyrmion_solver_b200``) never imports or calls it.

``initial_field(short, p_i, p_f, config)`` restates, vectorised over the
lattice, what the reference's ``Simulation.initialize`` (core/simulation.py:
124-172) leaves in ``Field`` for a theory's ``initial_config.initialize``
(th/<theory>/initial_config.py):

* modes ``ground`` / ``uniform`` / ``vacuum`` / ``gs``: create_ground_state_kernel
  (:792-857), components 0..3 = (1, 0, 0, 0);
* ``smorgasbord`` / ``smorgaasbord`` / ``smorg``: _initialize_smorgasbord
  (:1267-1407), seeded positions and Euler angles, rational-map lumps composed by
  normalised quaternion products from the vacuum;
* anything else: create_initial_configuration_kernel (:860-976) with the ansatz
  of the mode, the ``ansatz`` key or the parameters' flags: the Gaussian
  hedgehog (hedgehog_field :701-758), the rational map with the fitted profile
  (profilefun :342-442, rational_map_value :445-550), or the vacuum.

Theory differences (th/omega_skyrme and th/coulomb_skyrme initial_config.py:
52-72): the profile length of omega is 0.15 min(size) for both ansätze, that of
Coulomb 0.4 min(size) / max(|B|, 1); the others use r unscaled in the map and
max(size) / (8 max(|B|, 1)) in the hedgehog.  The ansatz flags sit at p_i[12:15]
for omega / Coulomb and p_i[11:14] otherwise; baryon number and isospin rotation
at p_f[11:13] for rho and p_f[10:12] otherwise; the smorgasbord's default count
reads p_f[10] for every theory.  Omega's seeded omega field (create_omega_field_kernel)
is not part of this function.

Pinned to the reference's own kernels run under Numba's CUDA simulator
(tests/golden/init.npz, made by tests/golden/make_golden_init.py).
"""
from __future__ import annotations

import math

import numpy as np

# profilefun's fitted coefficients: [B - 1][0 = massless, 1 = massive][a..e]
PROFILE = np.array([
    [[0.630647, 0.0218873, -0.0245431, 0.00300978, -0.00010542],
     [0.839091, -0.148868, 0.222428, -0.0900171, 0.0107864]],
    [[0.162388, 0.297889, -0.0878554, 0.00931881, -0.000317398],
     [0.219378, 0.485652, -0.154501, 0.0197873, -0.000774393]],
    [[-0.000352877, 0.324957, -0.0792377, 0.00740042, -0.000232486],
     [0.0354001, 0.502948, -0.13181, 0.0142808, -0.000509656]],
    [[-0.0469393, 0.294323, -0.0599714, 0.00457823, -0.000110399],
     [-0.0127361, 0.4427, -0.0941955, 0.00808476, -0.00024485]],
    [[-0.0575367, 0.187057, -0.00254209, -0.00580857, 0.000517839],
     [-0.0568381, 0.337281, -0.0167685, -0.010309, 0.00119672]],
    [[-0.0450119, 0.104984, 0.0347624, -0.0119037, 0.000864464],
     [-0.05592, 0.229393, 0.0498254, -0.0257167, 0.00248365]],
    [[-0.0383968, 0.0703267, 0.0464174, -0.0130402, 0.000887014],
     [-0.0575166, 0.196602, 0.056918, -0.0244016, 0.00219296]],
    [[-0.013271, -0.00611001, 0.0751757, -0.0170388, 0.0010835],
     [-0.0335398, 0.0655383, 0.135378, -0.0430527, 0.00381564]],
    [[0.00853506, -0.0576792, 0.0896121, -0.0181863, 0.00109042],
     [-0.0101412, -0.0285699, 0.181351, -0.0517179, 0.00441035]],
])

GROUND = ("ground", "uniform", "vacuum", "gs")
SMORGASBORD = ("smorgasbord", "smorgaasbord", "smorg")
RATIONAL = ("rational_map", "rational map", "rational-map")


def _fit(r, B, row):
    k = PROFILE[B - 1, row] if 1 <= B <= 9 else np.zeros(5)
    poly = r * (k[0] + r * (k[1] + r * (k[2] + r * (k[3] + r * k[4]))))
    return math.pi * (1.0 - np.tanh(np.abs(poly)))


def profile(r, B, m0):
    if m0 < 1.0:
        f = (1.0 - m0) * _fit(r, B, 0) + m0 * _fit(r, B, 1)
    else:
        f = _fit(r, B, 1)
    return np.where(r < 1.0e-6, math.pi, np.where(r > 15.0, 0.0, f))


def _pow(z, n):
    r = np.ones_like(z)
    for _ in range(n):
        r = r * z
    return r


def rational_map(z, B):
    """R_B(z) for complex arrays z (th/nuclear_skyrme/initial_config.py:445-550); powers by
    repeated products, as cpow_uint."""
    def div(a, b):
        den = b.real * b.real + b.imag * b.imag + 1.0e-18
        out = np.empty_like(a)
        out.real = (a.real * b.real + a.imag * b.imag) / den
        out.imag = (a.imag * b.real - a.real * b.imag) / den
        return out
    s3 = math.sqrt(3.0)
    if B == 1:
        return z
    if B == 2:
        return z * z
    if B == 3:
        z2 = z * z
        return div(1j * s3 * z2 - 1.0, z * (z2 - 1j * s3) + 1.0e-9)
    if B == 4:
        z4 = _pow(z, 4)
        t = 2j * s3 * z * z
        return div(z4 + t + 1.0, z4 - t + 1.0)
    if B == 5:
        a, b = 3.0660, 3.9334
        z2 = z * z
        z4 = _pow(z, 4)
        return div(z * (z4 + b * z2 + a), a * z4 - b * z2 + 1.0)
    if B == 6:
        a = 0.1585
        z4 = _pow(z, 4)
        return div(z4 + 1j * a, z * z * (1j * a * z4 + 1.0) + 1.0e-9)
    if B == 7:
        z2, z5, z7 = z * z, _pow(z, 5), _pow(z, 7)
        return div(z7 - 7.0 * z5 - 7.0 * z2 - 1.0, z7 + 7.0 * z5 - 7.0 * z2 + 1.0)
    if B == 8:
        a = 0.1352
        z6 = _pow(z, 6)
        return div(z6 - a, z * z * (a * z6 + 1.0) + 1.0e-9)
    return _pow(z, B)


def _rot_z(v, a):
    c, s = math.cos(a), math.sin(a)
    return np.stack([c * v[0] + s * v[1], -s * v[0] + c * v[1], v[2]])


def _rot_y(v, a):
    c, s = math.cos(a), math.sin(a)
    return np.stack([c * v[0] - s * v[2], v[1], s * v[0] + c * v[2]])


def _euler(v, a):
    return _rot_z(_rot_y(_rot_z(v, a[0]), a[1]), a[2])


def _normalise(v):
    s = np.sqrt((v * v).sum(axis=0))
    return np.where(s == 0.0, v, v / np.where(s == 0.0, 1.0, s))


def _qmul(a, b):
    return np.stack([a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3],
                     a[0] * b[1] + b[0] * a[1] + a[2] * b[3] - a[3] * b[2],
                     a[0] * b[2] + b[0] * a[2] + a[3] * b[1] - a[1] * b[3],
                     a[0] * b[3] + b[0] * a[3] + a[1] * b[2] - a[2] * b[1]])


def _grid(p_i, p_f):
    X, Y, Z = (int(v) for v in p_i[:3])
    h = [float(p_f[3]), float(p_f[4]), float(p_f[5])]
    gx, gy, gz = np.meshgrid(h[0] * np.arange(X, dtype=np.float64), h[1] * np.arange(Y, dtype=np.float64),
                             h[2] * np.arange(Z, dtype=np.float64), indexing="ij")
    centre = [0.5 * (0.0 + h[d] * float(n - 1)) for d, n in enumerate((X, Y, Z))]
    return np.stack([gx, gy, gz]), centre


def hedgehog(g, c, r0, rotation):
    r3 = np.stack([g[0] - c[0], g[1] - c[1], g[2] - c[2]])
    r = np.sqrt((r3 * r3).sum(axis=0))
    q = r / r0
    f = math.pi * np.exp(-(q * q))
    inv = 1.0 / np.where(r < 1.0e-12, 1.0, r)
    n = _rot_z(r3 * inv, rotation)
    out = np.concatenate([np.cos(f)[None], np.sin(f) * n])
    centre = r < 1.0e-12
    out[:, centre] = np.array([-1.0, 0.0, 0.0, 0.0])[:, None]
    return out


def map_lump(g, c, alpha, beta, B, r0, m0):
    r3 = _euler(np.stack([g[0] - c[0], g[1] - c[1], g[2] - c[2]]), alpha)
    r = np.sqrt((r3 * r3).sum(axis=0))
    Bi = max(int(abs(B) + 0.5), 1)
    small = r < 1.0e-6
    with np.errstate(invalid="ignore", divide="ignore"):
        theta = np.where(small, 0.0, np.arccos(r3[2] / np.where(small, 1.0, r)))
    ph = np.where(small, 0.0, np.arctan2(r3[1], r3[0]))
    t = np.tan(0.5 * theta)
    R = rational_map(np.cos(ph) * t + 1j * (np.sin(ph) * t), Bi)
    f = profile(r / r0, Bi, m0)
    a = R.real * R.real + R.imag * R.imag
    den = 1.0 + a
    n = _euler(np.stack([2.0 * R.real / den, 2.0 * R.imag / den, (1.0 - a) / den]), beta)
    return np.concatenate([np.cos(f)[None], n * np.sin(f)])


def _layout(short):
    if short in ("omega", "coulomb"):
        return 12, 10
    if short == "rho":
        return 11, 11
    return 11, 10


def _scales(short, B, p_f):
    size = [float(p_f[0]), float(p_f[1]), float(p_f[2])]
    if short == "omega":
        s = max(0.15 * min(size) / 1.0, 1.0e-6)
        return s, s
    if short == "coulomb":
        s = max(0.4 * min(size) / max(abs(B), 1.0), 1.0e-6)
        return s, s
    return max(max(size) / (8.0 * max(abs(B), 1.0)), 1.0e-6), 1.0


def initial_field(short, p_i, p_f, config=None):
    """(C, X, Y, Z) FP64 field the reference's initialize leaves (omega field not seeded)."""
    cfg = dict(config or {})
    p_i = np.asarray(p_i)
    p_f = np.asarray(p_f, np.float64)
    C = int(p_i[5])
    g, centre = _grid(p_i, p_f)
    shape = g.shape[1:]
    field = np.zeros((C,) + shape)
    field[0] = 1.0
    mode = str(cfg.get("mode", "initial")).lower().strip()
    if mode in GROUND:
        return field
    iflag, ib = _layout(short)
    if mode in SMORGASBORD:
        rng = np.random.default_rng(int(cfg.get("seed", 0)))
        size = [float(p_f[0]), float(p_f[1]), float(p_f[2])]
        count = int(cfg.get("count", max(1, int(round(abs(float(cfg.get("baryon_number", p_f[10]))))))))
        lump_b = int(cfg.get("lump_baryon", 1))
        m0 = float(cfg.get("profile_m0", 1.0))
        ps = float(cfg.get("position_scale", 0.18))
        d = [ps * s for s in size]
        pos = rng.uniform(low=[-d[0], -d[1], -d[2]], high=d, size=(count, 3))
        pos -= pos.mean(axis=0, keepdims=True)
        alphas = rng.uniform(0.0, 2.0 * math.pi, size=(count, 3))
        betas = rng.uniform(0.0, 2.0 * math.pi, size=(count, 3))
        _, r0 = _scales(short, float(lump_b), p_f)
        acc = field[:4].copy()
        for n in range(count):
            c = [float(centre[k] + pos[n, k]) for k in range(3)]
            v = _normalise(map_lump(g, c, alphas[n], betas[n], float(lump_b), r0, m0))
            acc = _normalise(_qmul(acc, v))
        field[:4] = acc
        return field
    ans = "hedgehog"
    if int(p_i[iflag + 1]) != 0:
        ans = "rational_map"
    elif int(p_i[iflag + 2]) != 0:
        ans = "uniform"
    if mode in RATIONAL:
        ans = "rational_map"
    else:
        ans = str(cfg.get("ansatz", ans)).lower().strip()
    B = float(cfg.get("baryon_number", p_f[ib]))
    iso = float(cfg.get("isospin_rotation", p_f[ib + 1]))
    r_hh, r_map = _scales(short, B, p_f)
    if ans in RATIONAL:
        v = map_lump(g, centre, (0.0, 0.0, 0.0), (0.0, 0.0, iso), B, r_map, 1.0)
    elif ans == "hedgehog":
        v = hedgehog(g, centre, r_hh, iso)
    else:
        return field
    field[:4] = _normalise(v)
    return field
