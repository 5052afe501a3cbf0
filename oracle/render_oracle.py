"""NumPy oracle for the viewer's volume builder and ray-march.

TEST INFRASTRUCTURE ONLY.  ``tests/`` and ``__graft_entry__.smoke()`` import
this module as the checker; the product (``skyrmion_solver_b200``) never
imports or calls it.

* ``rgba_volume`` restates build_rgba_volume_kernel with the extrema of
  _reduce_density_extrema (th/nuclear_skyrme/render_gl.py:157-222, 447-500) in
  FP64, stored as FP32.  It is pinned to the reference's own kernels run under
  Numba's CUDA simulator (tests/golden/volume.npz, made by
  tests/golden/make_golden_volume.py).
* ``inv_view_rows`` restates GLBackend._rotation_matrix / make_inv_view_rows
  (visualization/gl_backend.py:1166-1228).
* ``render`` restates the ray-march fragment shader
  (visualization/gl_backend.py:519-710) in FP32, vectorised over pixels, with
  the GL_LINEAR / GL_CLAMP_TO_EDGE filtering of the volume and transfer
  textures written out (texel centres at (i + 0.5) / n).  The shader itself
  runs only through OpenGL, which this machine does not have, so the image is
  not pinned to the reference's output; the restatement is checked against
  hand-derived cases in tests/test_render.py instead.
"""
from __future__ import annotations

import numpy as np

F = np.float32

# gl_backend.py:839
TRANSFER = np.array([[0.0, 0.0, 0.0, 0.0], [1.0, 0.0, 0.0, 1.0], [1.0, 0.5, 0.0, 1.0], [1.0, 1.0, 0.0, 1.0],
                     [0.0, 1.0, 0.0, 1.0], [0.0, 1.0, 1.0, 1.0], [0.0, 0.0, 1.0, 1.0], [1.0, 0.0, 1.0, 1.0],
                     [0.0, 0.0, 0.0, 0.0]], dtype=F)


def rgba_volume(density, field, dims):
    """(volume (Z, Y, X, 4) float32, min, max) from an FP64 density of N sites and a reference-layout field."""
    X, Y, Z = dims
    N = X * Y * Z
    d = np.asarray(density, np.float64).reshape(N)
    f = np.asarray(field, np.float64).reshape(-1, N)
    vmin, vmax = float(d.min()), float(d.max())
    dn = (d - vmin) / (vmax - vmin + 1.0e-30)
    p1, p2, p3 = f[1], f[2], f[3]
    n2 = p1 * p1 + p2 * p2 + p3 * p3
    small = n2 <= 1.0e-20
    inv = 1.0 / np.sqrt(np.where(small, 1.0, n2))
    nx = np.where(small, 0.0, p1 * inv)
    ny = np.where(small, 0.0, p2 * inv)
    nz = np.where(small, 1.0, p3 * inv)
    vol = np.stack([dn, nx, ny, nz], axis=-1).astype(F).reshape(X, Y, Z, 4)
    return np.ascontiguousarray(vol.transpose(2, 1, 0, 3)), vmin, vmax


def inv_view_rows(view_rotation=(0.0, 0.0, 0.0), view_translation=(0.0, 0.0, -4.0)):
    """The shader's three inverse-view rows (3, 4) float32."""
    rx = np.deg2rad(-float(view_rotation[0]))
    ry = np.deg2rad(-float(view_rotation[1]))
    cx, sx, cy, sy = np.cos(rx), np.sin(rx), np.cos(ry), np.sin(ry)
    rot_x = np.array([[1.0, 0.0, 0.0], [0.0, cx, -sx], [0.0, sx, cx]], dtype=F)
    rot_y = np.array([[cy, 0.0, sy], [0.0, 1.0, 0.0], [-sy, 0.0, cy]], dtype=F)
    rot = np.eye(4, dtype=F)
    rot[:3, :3] = rot_x @ rot_y
    trans = np.eye(4, dtype=F)
    trans[:3, 3] = [-float(v) for v in view_translation]
    return (rot @ trans)[:3].astype(F)


def _lin(s, n):
    u = s * F(n) - F(0.5)
    fl = np.floor(u)
    w = u - fl
    i = fl.astype(np.int64)
    return np.clip(i, 0, n - 1), np.clip(i + 1, 0, n - 1), w


def sample(vol, sx, sy, sz):
    """Trilinear clamp-to-edge lookup of a (Z, Y, X, 4) volume at normalised coordinates: (P, 4)."""
    Z, Y, X = vol.shape[:3]
    x0, x1, wx = _lin(sx, X)
    y0, y1, wy = _lin(sy, Y)
    z0, z1, wz = _lin(sz, Z)
    wx, wy, wz = wx[:, None], wy[:, None], wz[:, None]

    def lerp(a, b, t):
        return a + (b - a) * t
    c00 = lerp(vol[z0, y0, x0], vol[z0, y0, x1], wx)
    c10 = lerp(vol[z0, y1, x0], vol[z0, y1, x1], wx)
    c01 = lerp(vol[z1, y0, x0], vol[z1, y0, x1], wx)
    c11 = lerp(vol[z1, y1, x0], vol[z1, y1, x1], wx)
    return lerp(lerp(c00, c10, wy), lerp(c01, c11, wy), wz)


def transfer(s):
    i0, i1, w = _lin(s, TRANSFER.shape[0])
    return TRANSFER[i0] + (TRANSFER[i1] - TRANSFER[i0]) * w[:, None]


def pion_rgb(n):
    """pionVectorToRGB (gl_backend.py:573-592) for n of shape (P, 3)."""
    pi = F(3.14159265359)
    l = F(0.5) * (n[:, 2] + F(1.0))
    c = F(1.0) - np.abs(F(2.0) * l - F(1.0))
    h = np.arctan2(n[:, 1], n[:, 0]).astype(F)
    h = np.where(h < 0, h + F(2.0) * pi, h)
    hp = F(3.0) * h / pi
    md = hp - F(2.0) * np.floor(hp / F(2.0))
    x = c * (F(1.0) - np.abs(md - F(1.0)))
    m = l - F(0.5) * c
    out = np.zeros((n.shape[0], 3), F)
    for k, (r, g, b) in enumerate([(c + m, x + m, m), (x + m, c + m, m), (m, c + m, x + m),
                                   (m, x + m, c + m), (x + m, m, c + m), (c + m, m, x + m)]):
        sel = (hp >= k) & (hp < k + 1)
        out[sel] = np.stack([r, g, b], axis=1)[sel]
    return out


def render(vol, rows, box=(1.0, 1.0, 1.0), zoom=5.5, brightness=6.0, levelset=0.2, dmin=0.0, dmax=1.0,
           transfer_scale=4.0, opacity_scale=1.0, tstep=0.002, max_steps=2500, color_mode=0, width=64, height=48):
    """(height, width, 4) float32 RGBA, row 0 at the top; rays that miss the box are (1, 1, 1, 1)."""
    rows = np.asarray(rows, F)
    box = np.asarray(box, F)
    col = np.arange(width, dtype=F)
    row = np.arange(height, dtype=F)
    u = ((col + F(0.5)) / F(width)) * F(2.0) - F(1.0)
    v = (F(1.0) - (row + F(0.5)) / F(height)) * F(2.0) - F(1.0)
    U, V = np.meshgrid(u, v)
    U, V = U.ravel(), V.ravel()
    P = U.size
    o = rows[:, 3]
    p = np.stack([U, V, np.full(P, -F(zoom), F)], axis=1)
    d = p @ rows[:, :3].T
    d = d / np.sqrt((d * d).sum(axis=1))[:, None]
    with np.errstate(divide="ignore", invalid="ignore"):   # axis-parallel rays: 1 / 0 = inf, as in GLSL
        inv = F(1.0) / d
        tbot = inv * (-box - o)
        ttop = inv * (box - o)
    tnear = np.minimum(ttop, tbot).max(axis=1)
    tfar = np.maximum(ttop, tbot).min(axis=1)
    hit = tfar > tnear
    idx = np.nonzero(hit)[0]
    tnear = np.where(tnear < 0, F(0.0), tnear).astype(F)[idx]
    img = np.ones((P, 4), F)
    pos = o + d[idx] * tnear[:, None]
    stepv = d[idx] * F(tstep)
    t = tnear.copy()
    tf = tfar[idx]
    acc = np.zeros((idx.size, 4), F)
    live = np.ones(idx.size, bool)
    black = np.zeros(idx.size, bool)
    denom = F(max(F(dmax) - F(dmin), F(1.0e-30)))
    for _ in range(int(max_steps)):
        a = np.nonzero(live)[0]
        if a.size == 0:
            break
        q = pos[a]
        e = np.minimum(np.abs(q + box), np.abs(q - box))
        edge = (e < F(0.005)).sum(axis=1) >= 2
        black[a[edge]] = True
        live[a[edge]] = False
        a, q = a[~edge], q[~edge]
        tc = (q / box) * F(0.5) + F(0.5)
        sv = sample(vol, tc[:, 0], tc[:, 1], tc[:, 2])
        norm = (sv[:, 0] - F(dmin)) / denom
        inp = np.maximum((norm - F(levelset)) * F(transfer_scale), F(0.0))
        if color_mode == 0:
            c = transfer(np.clip(norm, F(0.0), F(1.0)))
            c[:, 3] *= F(opacity_scale)
        else:
            rgb = pion_rgb(sv[:, 1:4])
            c = np.concatenate([inp[:, None] * rgb, (inp * F(opacity_scale))[:, None]], axis=1)
        c[:, :3] *= c[:, 3:4]
        acc[a] = acc[a] + c * (F(1.0) - acc[a, 3:4])
        stop = acc[a, 3] > F(0.95)
        t[a] = t[a] + F(tstep)
        stop |= t[a] > tf[a]
        live[a[stop]] = False
        go = a[~stop]
        pos[go] = pos[go] + stepv[go]
    out = np.clip(acc * F(brightness), F(0.0), F(1.0))
    out[black] = np.array([0.0, 0.0, 0.0, 1.0], F)
    img[idx] = out
    return img.reshape(height, width, 4)
