"""Shared ``initialize`` implementation for the theory packages.

Builds the initial Skyrme field on the host in FP64 (``skyrmion_solver_b200.initial``)
and uploads it into the simulation's ``Field`` buffer.  Supported ``config`` keys:

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


def make_initialize(short):
    def initialize(*, Velocity, Field, grid=None, p_i_d=None, p_f_d=None, p_i_h=None, p_f_h=None, config=None,
                   **_unused):
        import torch
        cfg = config or {}
        p_i = np.asarray(p_i_h if p_i_h is not None else p_i_d.host)
        p_f = np.asarray(p_f_h if p_f_h is not None else p_f_d.host)
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
