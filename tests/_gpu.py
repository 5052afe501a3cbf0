"""GPU-test helpers: device buffers from the golden fixtures and a Simulation wired to them."""
import numpy as np

from skyrmion_solver_b200 import theories as T
from skyrmion_solver_b200.core.simulation import Simulation
from tests.golden.make_golden import theory_params


def dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64).ravel()).cuda()


def host(t, shape=None):
    a = t.detach().cpu().numpy()
    return a.reshape(shape) if shape is not None else a


def golden_simulation(name, d):
    th = T.by_short_name(name)
    sim = Simulation(theory_params(name, th), th)
    assert np.array_equal(sim.p_i_h, d["p_i"]) and np.array_equal(sim.p_f_h, d["p_f"])
    sim.Field.copy_(dev(d["field0"]))
    sim.Velocity.copy_(dev(d["velocity0"]))
    return th, sim
