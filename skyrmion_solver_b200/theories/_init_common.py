"""Shared ``initialize`` implementation for the theory packages.

Two families of initial fields are built, both in FP64 in the reference layout.

The reference's own configurations (th/<theory>/initial_config.py ``initialize``),
built on the device by ``sky_init_lumps``; this is what a configuration without
the keys below selects, exactly as the reference reads it:

* ``mode``: ``"ground"`` / ``"uniform"`` / ``"vacuum"`` / ``"gs"`` (vacuum),
  ``"smorgasbord"`` / ``"smorgaasbord"`` / ``"smorg"`` (seeded rational-map lumps
  composed by quaternion products; keys ``seed``, ``count``, ``lump_baryon``,
  ``profile_m0``, ``profile_m1``, ``position_scale``), ``"rational_map"``, or
  anything else (default ``"initial"``): the ansatz of the ``ansatz`` key or of
  the parameters' flags, a Gaussian hedgehog, a fitted-profile rational map or the
  vacuum;
* ``baryon_number``, ``isospin_rotation`` (default: the packed parameters);
* omega: the omega field is seeded as -c_omega B0 (create_omega_field_kernel,
  th/omega_skyrme/initial_config.py:1496-1533) except in the vacuum.

Synthetic workload fields (``build_device_field`` through ``sky_init_field``, or
``build_host_field`` in NumPy where noise or an explicit field is asked for):
selected by ``mode`` ``"product"``, ``"field"`` or ``"cloud"``, or by any of the
keys ``scale`` (profile f(r) = pi exp(-r/scale), default 1.5), ``center``,
``noise`` (seeded uniform amplitude added before renormalising),
``vacuum_shell`` (width of the boundary shell set to the vacuum), ``positions``,
``orientations``, ``min_separation``.  Modes there: ``"ground"``,
``"hedgehog"``, ``"rational_map"`` (B = 1, 2, 4), ``"product"`` (explicit
positions / orientations), ``"cloud"`` (``count`` seeded hedgehogs at random
positions with Haar orientations; ``"smorgasbord"`` with one of the keys above
means the same), ``"field"`` (explicit ``field``, optional ``velocity``).
Omega's field is seeded likewise unless ``omega_seed`` is False or the field is
explicit.
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
    elif mode in ("cloud", "smorgasbord"):
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
    if mode in ("cloud", "smorgasbord"):
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


GROUND_MODES = ("ground", "uniform", "vacuum", "gs")
SMORGASBORD_MODES = ("smorgasbord", "smorgaasbord", "smorg")
RATIONAL_MODES = ("rational_map", "rational map", "rational-map")
SYNTHETIC_MODES = ("product", "field", "cloud")
SYNTHETIC_KEYS = ("scale", "center", "noise", "vacuum_shell", "positions", "orientations", "min_separation")
LUMP_STRIDE = 16


def is_reference_config(config) -> bool:
    """True when the configuration asks for one of the reference's own initial fields."""
    cfg = config or {}
    mode = str(cfg.get("mode", "initial")).lower().strip()
    return mode not in SYNTHETIC_MODES and not any(k in cfg for k in SYNTHETIC_KEYS)


def _ansatz_slots(short):
    """(p_i index of the hedgehog flag, p_f index of the baryon number) of a theory's packing."""
    if short in ("omega", "coulomb"):
        return 12, 10
    if short == "rho":
        return 11, 11
    return 11, 10


def _profile_lengths(short, B, p_f):
    """(hedgehog r0, map radius divisor) of th/<theory>/initial_config.py: omega uses
    0.15 min(size) for both, Coulomb 0.4 min(size) / max(|B|, 1) for both; the others
    max(size) / (8 max(|B|, 1)) in the hedgehog and the unscaled radius in the map."""
    size = [float(p_f[0]), float(p_f[1]), float(p_f[2])]
    if short == "omega":
        s = max(0.15 * min(size) / 1.0, 1.0e-6)
        return s, s
    if short == "coulomb":
        s = max(0.4 * min(size) / max(abs(B), 1.0), 1.0e-6)
        return s, s
    return max(max(size) / (8.0 * max(abs(B), 1.0)), 1.0e-6), 1.0


def reference_lumps(short, p_i, p_f, config=None):
    """The lump list (n, 16) and the from-vacuum flag of the reference's initialize for this
    configuration (th/nuclear_skyrme/initial_config.py:1267-1560 and the theory's variant)."""
    cfg = dict(config or {})
    p_i = np.asarray(p_i)
    p_f = np.asarray(p_f, np.float64)
    X, Y, Z = (int(v) for v in p_i[:3])
    h = (float(p_f[3]), float(p_f[4]), float(p_f[5]))
    centre = [0.5 * (0.0 + h[d] * float(n - 1)) for d, n in enumerate((X, Y, Z))]   # _physical_box_center
    mode = str(cfg.get("mode", "initial")).lower().strip()
    if mode in GROUND_MODES:
        return np.zeros((0, LUMP_STRIDE)), True
    iflag, ib = _ansatz_slots(short)
    if mode in SMORGASBORD_MODES:
        rng = np.random.default_rng(int(cfg.get("seed", 0)))
        size = [float(p_f[0]), float(p_f[1]), float(p_f[2])]
        count = int(cfg.get("count", max(1, int(round(abs(float(cfg.get("baryon_number", p_f[10]))))))))
        lump_b = int(cfg.get("lump_baryon", 1))
        m0 = float(cfg.get("profile_m0", 1.0))
        scale = float(cfg.get("position_scale", 0.18))
        half = [scale * v for v in size]
        pos = rng.uniform(low=[-half[0], -half[1], -half[2]], high=half, size=(count, 3))
        pos -= pos.mean(axis=0, keepdims=True)
        alpha = rng.uniform(0.0, 2.0 * np.pi, size=(count, 3))
        beta = rng.uniform(0.0, 2.0 * np.pi, size=(count, 3))
        _, r_map = _profile_lengths(short, float(lump_b), p_f)
        lumps = np.zeros((count, LUMP_STRIDE))
        for n in range(count):
            lumps[n, 0] = 1.0
            lumps[n, 1] = float(lump_b)
            lumps[n, 2:5] = [float(centre[d] + pos[n, d]) for d in range(3)]
            lumps[n, 5:8] = alpha[n]
            lumps[n, 8:11] = beta[n]
            lumps[n, 11] = r_map
            lumps[n, 12] = m0
        return lumps, True
    ans = "hedgehog"
    if int(p_i[iflag + 1]) != 0:
        ans = "rational_map"
    elif int(p_i[iflag + 2]) != 0:
        ans = "uniform"
    ans = "rational_map" if mode in RATIONAL_MODES else str(cfg.get("ansatz", ans)).lower().strip()
    B = float(cfg.get("baryon_number", p_f[ib]))
    iso = float(cfg.get("isospin_rotation", p_f[ib + 1]))
    r_hh, r_map = _profile_lengths(short, B, p_f)
    lump = np.zeros((1, LUMP_STRIDE))
    lump[0, 1] = B
    lump[0, 2:5] = centre
    lump[0, 10] = iso
    if ans in RATIONAL_MODES:
        lump[0, 0], lump[0, 11], lump[0, 12] = 1.0, r_map, 1.0
    elif ans == "hedgehog":
        lump[0, 0], lump[0, 11] = 0.0, r_hh
    else:
        return np.zeros((0, LUMP_STRIDE)), True
    return lump, False


def build_reference_field(short, p_i, p_f, config, out, stream=None):
    """Write the reference's initial field for `config` into `out` (FP64 CUDA tensor of C*N
    values) with sky_init_lumps; omega's field component is left at 0."""
    from .. import _lib
    p_i = np.ascontiguousarray(p_i, np.int32)
    p_f = np.ascontiguousarray(p_f, np.float64)
    lumps, from_vacuum = reference_lumps(short, p_i, p_f, config)
    lumps = np.ascontiguousarray(lumps, np.float64)
    _lib.call("sky_init_lumps", _lib.i32p(p_i), len(p_i), _lib.f64p(p_f), len(p_f), len(lumps), _lib.f64p(lumps),
              1 if from_vacuum else 0, _lib.dptr(out), _lib.stream_ptr(stream))
    return out


def _host_params(p_i_d, p_f_d):
    """Host copies of device parameter arrays (DeviceParams, Numba device arrays or tensors)."""
    from .. import _lib
    return _lib.host_params(p_i_d, p_f_d)


def _as_tensor(buf):
    """A torch view of a device buffer: torch tensors as they are, other objects with a
    __cuda_array_interface__ (Numba device arrays from the reference's Simulation) zero-copy."""
    import torch
    if buf is None or isinstance(buf, torch.Tensor):
        return buf
    if hasattr(buf, "__cuda_array_interface__"):
        return torch.as_tensor(buf, device="cuda")
    return buf


def make_initialize(short):
    def initialize(*, Velocity, Field, grid=None, p_i_d=None, p_f_d=None, p_i_h=None, p_f_h=None, config=None,
                   **_unused):
        import torch
        Field, Velocity = _as_tensor(Field), _as_tensor(Velocity)
        _unused = {k: _as_tensor(v) if k in ("k1", "k2", "k3", "k4", "l1", "l2", "l3", "l4", "Temp") else v
                   for k, v in _unused.items()}
        cfg = config or {}
        hi, hf = _host_params(p_i_d if p_i_h is None else None, p_f_d if p_f_h is None else None)
        p_i = np.asarray(p_i_h if p_i_h is not None else hi)
        p_f = np.asarray(p_f_h if p_f_h is not None else hf)
        mode = str(cfg.get("mode", "initial")).lower().strip()
        if is_reference_config(cfg):
            if not Field.is_cuda:
                raise RuntimeError("the reference's initial configurations are built on a CUDA device")
            build_reference_field(short, p_i, p_f, cfg, Field)
            Velocity.zero_()
            for name in ("k1", "k2", "k3", "k4", "l1", "l2", "l3", "l4", "Temp"):   # zeroed as the reference's kernels do
                buf = _unused.get(name)
                if buf is not None and hasattr(buf, "zero_"):
                    buf.zero_()
            seed = short == "omega" and mode not in GROUND_MODES
        else:
            if Field.is_cuda and not float(cfg.get("noise", 0.0)) and mode != "field":
                # built in place on the device (sky_init_field); noise and explicit fields come from the host
                Field.copy_(build_device_field(short, p_i, p_f, cfg, Field.device.index or 0))
            else:
                f = build_host_field(short, p_i, p_f, cfg)
                Field.copy_(torch.from_numpy(f.ravel()).to(Field.device))
            seed = short == "omega" and cfg.get("omega_seed", True) and mode != "field"
        if "velocity" in cfg:
            v = np.asarray(cfg["velocity"], dtype=np.float64).ravel()
            Velocity.copy_(torch.from_numpy(v).to(Velocity.device))
        if seed:
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
