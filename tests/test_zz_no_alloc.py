"""The allocation-free arrested-Newton step (sky_arrested_newton_step_noalloc).

Some callers cannot allocate device memory: a plugin that is handed only the
field and velocity of a host application whose allocator owns the device, or
an interactive loop that must not call cudaMalloc / cudaFree between frames
because they synchronise the device.  For them the library offers a step whose
working memory (the RK4 slopes, the stage field and the reduction scratch) is a
static device array of the library.  This file checks, through the C ABI, that
two consecutive calls give the same energy, err, field, velocity and gradient
as the allocating entry point (1e-10 relative, the tolerance of the step parity
tests), and that a lattice too large for the static array is refused.  It is
collected last on purpose so that a run stopping at the first failure has
already run every other test.
"""
import ctypes

import numpy as np
import pytest

from tests import _golden as G

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-10


def _dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64).ravel()).cuda()


# Largest value count C*N the static array admits, and lattices at and above it:
# 9 C N + 2 * 2376 doubles of working memory in 2 Mi doubles.
MAX_VALUES = 232488


def _compare_steps(name, p_i, p_f, field0, velocity0, energy0):
    """Two calls in a row of both entry points from the same state, compared."""
    import torch
    from skyrmion_solver_b200 import _lib
    from skyrmion_solver_b200._lib import THEORY_IDS, f64p, i32p
    from skyrmion_solver_b200.core.utils import scratch_doubles
    p_i = np.ascontiguousarray(p_i, np.int32)
    p_f = np.ascontiguousarray(p_f, np.float64)
    tid = THEORY_IDS[name]
    # allocating entry point: caller-provided slopes, stage field and scratch
    Fa, Va = _dev(field0), _dev(velocity0)
    EGa = torch.zeros_like(Fa)
    bufs = [torch.zeros_like(Fa) for _ in range(9)]
    scratch = torch.zeros(2 * scratch_doubles(), dtype=torch.float64, device="cuda")
    # allocation-free entry point: only field, velocity and gradient
    Fb, Vb = _dev(field0), _dev(velocity0)
    EGb = torch.zeros_like(Fb)
    torch.cuda.synchronize()
    stream = _lib.stream_ptr()
    prev_a = prev_b = float(energy0)
    for call in range(2):
        ea, erra = ctypes.c_double(), ctypes.c_double()
        _lib.call("sky_arrested_newton_step", tid, i32p(p_i), len(p_i), f64p(p_f), len(p_f), _lib.dptr(Va),
                  _lib.dptr(Fa), _lib.dptr(EGa), *[_lib.dptr(b) for b in bufs], _lib.dptr(scratch),
                  scratch.numel(), prev_a, ctypes.byref(ea), ctypes.byref(erra), stream)
        eb, errb = ctypes.c_double(), ctypes.c_double()
        _lib.call("sky_arrested_newton_step_noalloc", tid, i32p(p_i), len(p_i), f64p(p_f), len(p_f),
                  _lib.dptr(Vb), _lib.dptr(Fb), _lib.dptr(EGb), prev_b, ctypes.byref(eb), ctypes.byref(errb),
                  stream)
        torch.cuda.synchronize()
        assert abs(eb.value - ea.value) <= STEP_TOL * abs(ea.value), (call, eb.value, ea.value)
        assert abs(errb.value - erra.value) <= STEP_TOL * max(1.0, abs(erra.value)), (call, errb.value, erra.value)
        for a, b in ((Fa, Fb), (EGa, EGb)):
            assert G.rel_err(b.cpu().numpy(), a.cpu().numpy()) <= STEP_TOL
        va, vb = Va.cpu().numpy(), Vb.cpu().numpy()
        if np.any(va):
            assert G.rel_err(vb, va) <= STEP_TOL
        else:
            assert not np.any(vb)
        prev_a, prev_b = ea.value, eb.value


@pytest.mark.parametrize("name", ["nuclear", "omega", "rho"])
def test_noalloc_step_matches_allocating_step(name):
    d = G.load(name)
    _compare_steps(name, d["p_i"], d["p_f"], d["field0"], d["velocity0"], d["energy0"])


def _limit_case(name, dims, seed):
    """A seeded off-vacuum field on a lattice of the given dims (hedgehog with noise for the
    pion components, small seeded values for the others), its parameters and energy."""
    from skyrmion_solver_b200 import initial, theories as T
    th = T.by_short_name(name)
    p = th.params.default_params(xlen=dims[0], ylen=dims[1], zlen=dims[2], lsx=0.2, lsy=0.2, lsz=0.2,
                                 time_step=0.04)
    p_i, p_f = th.params.pack_device_params(p.resolved())
    C = int(p_i[5])
    rng = np.random.default_rng(seed)
    F = np.zeros((C,) + tuple(dims))
    F[:4] = initial.hedgehog(dims, (0.2, 0.2, 0.2), initial.exp_profile(1.0))
    F[:4] += rng.uniform(-1e-3, 1e-3, size=F[:4].shape)
    F[:4] /= np.sqrt((F[:4] ** 2).sum(axis=0))
    if C > 4:
        F[4:] = rng.uniform(-1e-2, 1e-2, size=F[4:].shape)
    V = np.zeros_like(F)
    return p_i, p_f, F, V


def test_noalloc_step_at_the_size_limit():
    """omega on 18 x 41 x 63: C*N = 232,470 values, whose working memory ends 170 doubles
    short of the static array's end (the reduction counters sit in its last slots)."""
    import torch
    from skyrmion_solver_b200 import _lib
    from skyrmion_solver_b200._lib import THEORY_IDS, f64p, i32p
    dims = (18, 41, 63)
    assert 5 * dims[0] * dims[1] * dims[2] <= MAX_VALUES
    p_i, p_f, F, V = _limit_case("omega", dims, seed=3)
    p_i32 = np.ascontiguousarray(p_i, np.int32)
    p_f64 = np.ascontiguousarray(p_f, np.float64)
    from skyrmion_solver_b200.core.utils import scratch_doubles
    e0 = ctypes.c_double()
    Fd = _dev(F)
    scratch = torch.zeros(scratch_doubles(), dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    _lib.call("sky_total_energy", THEORY_IDS["omega"], i32p(p_i32), len(p_i32), f64p(p_f64), len(p_f64),
              _lib.dptr(Fd), _lib.dptr(scratch), scratch.numel(), ctypes.byref(e0), _lib.stream_ptr())
    _compare_steps("omega", p_i, p_f, F, V, e0.value)


def test_noalloc_step_rejects_one_lattice_past_the_limit():
    """nuclear on 13 x 17 x 263: C*N = 232,492 values, four more than the array admits."""
    import torch
    from skyrmion_solver_b200 import _lib, theories as T
    from skyrmion_solver_b200._lib import THEORY_IDS, SkyInvalidArgument, f64p, i32p
    th = T.by_short_name("nuclear")
    p = th.params.default_params(xlen=13, ylen=17, zlen=263, lsx=0.2, lsy=0.2, lsz=0.2)
    p_i, p_f = th.params.pack_device_params(p.resolved())
    p_i = np.ascontiguousarray(p_i, np.int32)
    p_f = np.ascontiguousarray(p_f, np.float64)
    assert 4 * 13 * 17 * 263 == MAX_VALUES + 4
    small = torch.zeros(16, dtype=torch.float64, device="cuda")   # never touched: the size check comes first
    e, err = ctypes.c_double(), ctypes.c_double()
    with pytest.raises(SkyInvalidArgument, match="too large for the allocation-free step"):
        _lib.call("sky_arrested_newton_step_noalloc", THEORY_IDS["nuclear"], i32p(p_i), len(p_i), f64p(p_f),
                  len(p_f), _lib.dptr(small), _lib.dptr(small), _lib.dptr(small), 0.0, ctypes.byref(e),
                  ctypes.byref(err), _lib.stream_ptr())


def test_noalloc_step_rejects_large_lattice():
    import torch
    from skyrmion_solver_b200 import _lib, theories as T
    from skyrmion_solver_b200._lib import THEORY_IDS, SkyInvalidArgument, f64p, i32p
    th = T.by_short_name("omega")
    p = th.params.default_params(xlen=64, ylen=64, zlen=64, lsx=0.2, lsy=0.2, lsz=0.2)
    p_i, p_f = th.params.pack_device_params(p.resolved())
    p_i = np.ascontiguousarray(p_i, np.int32)
    p_f = np.ascontiguousarray(p_f, np.float64)
    small = torch.zeros(16, dtype=torch.float64, device="cuda")   # never touched: the size check comes first
    e, err = ctypes.c_double(), ctypes.c_double()
    with pytest.raises(SkyInvalidArgument, match="too large for the allocation-free step"):
        _lib.call("sky_arrested_newton_step_noalloc", THEORY_IDS["omega"], i32p(p_i), len(p_i), f64p(p_f),
                  len(p_f), _lib.dptr(small), _lib.dptr(small), _lib.dptr(small), 0.0, ctypes.byref(e),
                  ctypes.byref(err), _lib.stream_ptr())
