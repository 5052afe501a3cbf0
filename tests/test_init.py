"""Initial fields built on the device (sky_init_field) against the host builders.

The host builders (skyrmion_solver_b200.initial) restate the reference's initial
configurations in NumPy; the device kernel computes the same fields in FP64 with
CUDA's transcendental functions, so the two agree to a few units in the last
place (tolerance 1e-12 absolute on unit-length fields).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CONFIGS = [
    {"mode": "ground"},
    {"mode": "hedgehog", "scale": 1.2, "center": (0.3, -0.2, 0.1)},
    {"mode": "rational_map", "baryon_number": 2, "scale": 1.5},
    {"mode": "rational_map", "baryon_number": 4, "scale": 2.0, "vacuum_shell": 2},
    {"mode": "product", "positions": [(-1.0, 0.0, 0.2), (1.1, 0.3, -0.4)],
     "orientations": [None, (0.5, 0.5, 0.5, 0.5)]},
    {"mode": "cloud", "count": 3, "seed": 7, "vacuum_shell": 2},
]


@pytest.mark.parametrize("cfg", CONFIGS, ids=lambda c: c["mode"] + str(c.get("baryon_number", c.get("count", ""))))
@pytest.mark.parametrize("name", ["nuclear", "omega"])
def test_device_field_matches_host(cfg, name):
    import torch
    from skyrmion_solver_b200 import theories as T
    from skyrmion_solver_b200.theories._init_common import build_device_field, build_host_field
    dims, h = (23, 30, 27), 0.2
    th = T.by_short_name(name)
    p = th.params.default_params(xlen=dims[0], ylen=dims[1], zlen=dims[2], lsx=h, lsy=h, lsz=h,
                                 xsize=h * (dims[0] - 1), ysize=h * (dims[1] - 1), zsize=h * (dims[2] - 1))
    p_i, p_f = th.params.pack_device_params(p.resolved())
    p_i, p_f = np.asarray(p_i, np.int32), np.asarray(p_f, np.float64)
    host = build_host_field(name, p_i, p_f, cfg)
    dev = build_device_field(name, p_i, p_f, cfg)
    torch.cuda.synchronize()
    got = dev.cpu().numpy().reshape(host.shape)
    assert np.max(np.abs(got - host)) <= 1e-12


def test_initialize_builds_on_the_device_and_keeps_the_host_path_for_noise():
    import torch
    from skyrmion_solver_b200 import theories as T
    from skyrmion_solver_b200.core.simulation import Simulation
    from skyrmion_solver_b200.theories._init_common import build_host_field
    th = T.by_short_name("nuclear")
    p = th.params.default_params(xlen=20, ylen=20, zlen=20, lsx=0.2, lsy=0.2, lsz=0.2)
    for cfg in ({"mode": "rational_map", "baryon_number": 2, "scale": 1.5},
                {"mode": "hedgehog", "noise": 1e-3, "seed": 3}):
        sim = Simulation(p, th)
        sim.initialize(cfg)
        torch.cuda.synchronize()
        host = build_host_field("nuclear", sim.p_i_h, sim.p_f_h, cfg)
        got = sim.Field.cpu().numpy().reshape(host.shape)
        assert np.max(np.abs(got - host)) <= 1e-12
