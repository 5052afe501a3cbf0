"""Host-side (FP64 NumPy) builders of initial Skyrme fields.

Conventions follow the reference's initial configurations
(skyrmion_solver th/nuclear_skyrme/initial_config.py):
  * coordinates are centred, x_i = h*i - (L-1)h/2 (:664-698);
  * stereographic coordinate z = tan(theta/2) e^{i phi} (:941-953) and
    n = (2 Re R, 2 Im R, 1 - |R|^2) / (1 + |R|^2) (zton, :284-306);
  * phi = (cos f, sin f n) (:583-587);
  * products of Skyrme fields are quaternion products (:591-627).
The fields are built once per solve (not timed) and uploaded to the device.
"""
from __future__ import annotations

import math

import numpy as np


def coords(dims, h, center=(0.0, 0.0, 0.0)):
    X, Y, Z = dims
    hx, hy, hz = h
    xs = (np.arange(X) - (X - 1) / 2.0) * hx - center[0]
    ys = (np.arange(Y) - (Y - 1) / 2.0) * hy - center[1]
    zs = (np.arange(Z) - (Z - 1) / 2.0) * hz - center[2]
    return np.meshgrid(xs, ys, zs, indexing="ij")


def exp_profile(scale):
    """f(r) = pi exp(-r / scale)."""
    return lambda r: math.pi * np.exp(-r / scale)


def hedgehog(dims, h, profile, center=(0.0, 0.0, 0.0)):
    """phi = (cos f, sin f x/r) as an array of shape (4, X, Y, Z)."""
    x, y, z = coords(dims, h, center)
    r = np.sqrt(x * x + y * y + z * z)
    f = profile(r)
    rs = np.where(r > 0.0, r, 1.0)
    s = np.sin(f)
    out = np.empty((4,) + tuple(dims))
    out[0] = np.cos(f)
    out[1] = np.where(r > 0.0, s * x / rs, 0.0)
    out[2] = np.where(r > 0.0, s * y / rs, 0.0)
    out[3] = np.where(r > 0.0, s * z / rs, 0.0)
    return out


def rational_map_value(zc, B):
    """R(z) for the symmetric rational maps used here (th/nuclear_skyrme/initial_config.py:446-549)."""
    if B == 1:
        return zc
    if B == 2:
        return zc * zc
    if B == 4:  # cubic map (z^4 + 2 sqrt3 i z^2 + 1) / (z^4 - 2 sqrt3 i z^2 + 1)
        t = 2.0 * math.sqrt(3.0) * 1j * zc * zc
        z4 = zc ** 4
        return (z4 + t + 1.0) / (z4 - t + 1.0)
    raise ValueError(f"rational map for B={B} is not provided")


def rational_map(dims, h, B, profile, center=(0.0, 0.0, 0.0)):
    """phi = (cos f, sin f n(R(z))) with z the stereographic angle coordinate."""
    x, y, z = coords(dims, h, center)
    r = np.sqrt(x * x + y * y + z * z)
    rs = np.where(r < 1.0e-6, 1.0, r)
    theta = np.where(r < 1.0e-6, 0.0, np.arccos(np.clip(z / rs, -1.0, 1.0)))
    ph = np.where(r < 1.0e-6, 0.0, np.arctan2(y, x))
    t = np.tan(0.5 * theta)
    zc = t * np.exp(1j * ph)
    R = rational_map_value(zc, B)
    a = np.abs(R) ** 2
    den = 1.0 + a
    n = (2.0 * R.real / den, 2.0 * R.imag / den, (1.0 - a) / den)
    f = profile(r)
    s = np.sin(f)
    return np.stack([np.cos(f), s * n[0], s * n[1], s * n[2]])


def quat_mul(a, b):
    """Quaternion product of two (4, ...) fields (th/nuclear_skyrme/initial_config.py:591-627)."""
    a0, a1, a2, a3 = a
    b0, b1, b2, b3 = b
    return np.stack([a0 * b0 - a1 * b1 - a2 * b2 - a3 * b3,
                     a0 * b1 + b0 * a1 + a2 * b3 - a3 * b2,
                     a0 * b2 + b0 * a2 + a3 * b1 - a1 * b3,
                     a0 * b3 + b0 * a3 + a1 * b2 - a2 * b1])


def isorotate(phi, q):
    """phi -> q phi q^-1 for a unit quaternion q (acts on the pion components)."""
    q = np.asarray(q, dtype=np.float64)
    qc = np.array([q[0], -q[1], -q[2], -q[3]])
    shape = (4,) + (1,) * (phi.ndim - 1)
    return quat_mul(quat_mul(q.reshape(shape) * np.ones_like(phi), phi), qc.reshape(shape) * np.ones_like(phi))


def haar_su2(rng):
    """Haar-random SU(2) element: a normalised 4-D Gaussian."""
    v = rng.standard_normal(4)
    return v / np.linalg.norm(v)


def normalise(phi):
    n = np.sqrt((phi[:4] ** 2).sum(axis=0))
    phi[:4] /= np.where(n > 0.0, n, 1.0)
    return phi


def vacuum_shell(phi, width=2):
    """Set the outer `width` sites of every face to the vacuum (1, 0, 0, 0, 0...)."""
    for ax in range(3):
        for sl in (slice(0, width), slice(-width, None)):
            idx = [slice(None)] * 4
            idx[ax + 1] = sl
            phi[tuple(idx)] = 0.0
            idx0 = list(idx)
            idx0[0] = 0
            phi[tuple(idx0)] = 1.0
    return phi


def product_ansatz(dims, h, positions, orientations, profile):
    """Quaternion product of B=1 hedgehogs at `positions` with isorotations `orientations`."""
    out = None
    for pos, q in zip(positions, orientations):
        s = hedgehog(dims, h, profile, center=pos)
        if q is not None:
            s = isorotate(s, q)
        out = s if out is None else quat_mul(out, s)
    return normalise(out)


def seeded_positions(rng, B, box, min_sep=2.0, frac=0.6, max_tries=100000):
    """Rejection-sample B centres with pairwise separation >= min_sep inside the central `frac` of `box`."""
    pos = []
    half = 0.5 * frac * np.asarray(box, dtype=np.float64)
    tries = 0
    while len(pos) < B:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("could not place the requested number of skyrmions")
        c = rng.uniform(-half, half)
        if all(np.linalg.norm(c - p) >= min_sep for p in pos):
            pos.append(c)
    return [tuple(p) for p in pos]


def with_extra_components(phi4, C, extra=None):
    """Pad a (4, ...) Skyrme field with C-4 extra components (zero unless given)."""
    out = np.zeros((C,) + phi4.shape[1:])
    out[:4] = phi4
    if extra is not None:
        out[4:] = extra
    return out
