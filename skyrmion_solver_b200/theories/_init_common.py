"""Shared ``initialize`` implementation for the theory packages.

Builds the initial Skyrme field in FP64: on the device by ``sky_init_field``
(``build_device_field``), or on the host (``skyrmion_solver_b200.initial``,
``build_host_field``) for configurations with noise or an explicit field, and
writes it into the simulation's ``Field`` buffer.  Supported ``config`` keys:

* ``mode``: ``"ground"`` (vacuum), ``"hedgehog"``, ``"rational_map"``,
  ``"product"`` (explicit ``positions`` / ``orientations``), ``"smorgasbord"``
  (``count`` seeded hedgehogs at random positions with Haar orientations) or
  ``"field"`` (an explicit ``field`` array, optional ``velocity``);
* ``scale`` (profile f(r) = pi exp(-r/scale), default 1.5), ``baryon_number``,
  ``center``, ``seed``, ``min_separation``;
* ``noise`` (uniform amplitude added before renormalising, seeded),
  ``vacuum_shell`` (width of the boundary shell set to the vacuum);
* omega theory: ``omega_seed`` (default True) sets omega = -c_omega B0, as the
  reference's create_omega_field_kernel (th/omega_skyrme/initial_config.py:1496-1533).
"""
from __future__ import annotations

import numpy as np

from .. import initial as ini


def build_host_field(short, p_i, p_f, config):
    X, Y, Z = (int(v) for v in p_i[:3])
    C = int(p_i[5])
    h = (float(p_f[3]), float(p_f[4]), float(p_f[5]))
    dims = (X, Y, Z)
    mode = str(config.get("mode", "ground")).lower()
    scale = float(config.get("scale", 1.5))
    prof = ini.exp_profile(scale)
    rng = np.random.default_rng(config.get("seed", 0))
    center = tuple(config.get("center", (0.0, 0.0, 0.0)))
    if mode in ("ground", "vacuum", "uniform"):
        phi = np.zeros((4,) + dims)
        phi[0] = 1.0
    elif mode == "hedgehog":
        phi = ini.hedgehog(dims, h, prof, center)
    elif mode in ("rational_map", "rational map", "rational-map"):
        phi = ini.rational_map(dims, h, int(config.get("baryon_number", 1)), prof, center)
    elif mode == "product":
        phi = ini.product_ansatz(dims, h, config["positions"], config.get("orientations",
                                 [None] * len(config["positions"])), prof)
    elif mode == "smorgasbord":
        B = int(config.get("count", config.get("baryon_number", 1)))
        box = (X * h[0], Y * h[1], Z * h[2])
        pos = ini.seeded_positions(rng, B, box, float(config.get("min_separation", 2.0)))
        qs = [ini.haar_su2(rng) for _ in range(B)]
        phi = ini.product_ansatz(dims, h, pos, qs, prof)
    elif mode == "field":
        f = np.asarray(config["field"], dtype=np.float64).reshape((C,) + dims)
        return f.copy()
    else:
        raise ValueError(f"unknown initial configuration mode '{mode}'")
    noise = float(config.get("noise", 0.0))
    if noise:
        phi = phi + rng.uniform(-noise, noise, size=phi.shape)
    phi = ini.normalise(phi)
    field = ini.with_extra_components(phi, C)
    w = int(config.get("vacuum_shell", 0))
    if w:
        ini.vacuum_shell(field, w)
    return field


def _soliton_list(X, Y, Z, h, config, rng):
    """(baryon numbers, centres, quaternions) of the configuration, drawn from `rng` in the
    same order as build_host_field draws them."""
    mode = str(config.get("mode", "ground")).lower()
    center = tuple(config.get("center", (0.0, 0.0, 0.0)))
    if mode in ("ground", "vacuum", "uniform"):
        return [], [], []
    if mode == "hedgehog":
        return [1], [center], [None]
    if mode in ("rational_map", "rational map", "rational-map"):
        B = int(config.get("baryon_number", 1))
        if B not in (1, 2, 4):
            raise ValueError(f"rational map for B={B} is not provided")
        return [B], [center], [None]
    if mode == "product":
        pos = list(config["positions"])
        qs = list(config.get("orientations", [None] * len(pos)))
        return [1] * len(pos), pos, qs
    if mode == "smorgasbord":
        B = int(config.get("count", config.get("baryon_number", 1)))
        box = (X * h[0], Y * h[1], Z * h[2])
        pos = ini.seeded_positions(rng, B, box, float(config.get("min_separation", 2.0)))
        qs = [ini.haar_su2(rng) for _ in range(B)]
        return [1] * B, pos, qs
    raise ValueError(f"unknown initial configuration mode '{mode}' for the device builder")


def build_device_field(short, p_i, p_f, config, device=0, stream=None):
    """The field of build_host_field, built on the device by sky_init_field (FP64, reference
    layout, flattened torch tensor of C*N values).  Configurations with ``noise`` or an explicit
    ``field`` are host-side inputs: build those with build_host_field."""
    import torch
    from .. import _lib
    if float(config.get("noise", 0.0)) or str(config.get("mode", "ground")).lower() == "field":
        raise ValueError("noise and explicit fields are built on the host (build_host_field)")
    p_i = np.asarray(p_i, np.int32)
    p_f = np.asarray(p_f, np.float64)
    X, Y, Z = (int(v) for v in p_i[:3])
    C = int(p_i[5])
    h = (float(p_f[3]), float(p_f[4]), float(p_f[5]))
    rng = np.random.default_rng(config.get("seed", 0))
    bs, pos, qs = _soliton_list(X, Y, Z, h, config, rng)
    n = len(bs)
    baryon = np.asarray(bs if n else [1], np.int32)
    centers = np.asarray([tuple(c) for c in pos] if n else [(0.0, 0.0, 0.0)], np.float64).reshape(-1)
    quats = np.asarray([(1.0, 0.0, 0.0, 0.0) if q is None else tuple(q) for q in qs] if n else [(1.0, 0.0, 0.0, 0.0)],
                       np.float64).reshape(-1)
    out = torch.empty(C * X * Y * Z, dtype=torch.float64, device=torch.device("cuda", device))
    _lib.call("sky_init_field", _lib.i32p(p_i), len(p_i), _lib.f64p(p_f), len(p_f), n, _lib.i32p(baryon),
              _lib.f64p(centers), _lib.f64p(quats), float(config.get("scale", 1.5)),
              int(config.get("vacuum_shell", 0)), _lib.dptr(out), _lib.stream_ptr(stream))
    return out


def make_initialize(short):
    def initialize(*, Velocity, Field, grid=None, p_i_d=None, p_f_d=None, p_i_h=None, p_f_h=None, config=None,
                   **_unused):
        import torch
        cfg = config or {}
        p_i = np.asarray(p_i_h if p_i_h is not None else p_i_d.host)
        p_f = np.asarray(p_f_h if p_f_h is not None else p_f_d.host)
        if Field.is_cuda and not float(cfg.get("noise", 0.0)) and str(cfg.get("mode", "ground")).lower() != "field":
            # built in place on the device (sky_init_field); noise and explicit fields come from the host
            Field.copy_(build_device_field(short, p_i, p_f, cfg, Field.device.index or 0))
        else:
            f = build_host_field(short, p_i, p_f, cfg)
            Field.copy_(torch.from_numpy(f.ravel()).to(Field.device))
        if "velocity" in cfg:
            v = np.asarray(cfg["velocity"], dtype=np.float64).ravel()
            Velocity.copy_(torch.from_numpy(v).to(Velocity.device))
        if short == "omega" and cfg.get("omega_seed", True) and cfg.get("mode", "ground") != "field":
            seed_omega(Field, p_i, p_f)
    return initialize


def seed_omega(Field, p_i, p_f):
    """omega = -c_omega * B0 density (th/omega_skyrme/initial_config.py:1496-1533)."""
    import torch
    from ..core.launch import DensityKernel
    N = int(p_i[6])
    comp = int(p_i[11])
    en = torch.zeros(N, dtype=torch.float64, device=Field.device)
    DensityKernel(1, 1, "baryon")(en, Field, None, p_i, p_f)
    Field[comp * N:(comp + 1) * N] = -float(p_f[9]) * en / float(p_f[6])
