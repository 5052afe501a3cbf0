"""The C-ABI library loads and exports every symbol the public header declares.
Only argument validation is exercised here (it returns before any CUDA call)."""
import ctypes

import numpy as np

from skyrmion_solver_b200 import _lib


def test_header_symbols_exported():
    lib = _lib.load()
    syms = _lib.header_symbols()
    assert len(syms) >= 18
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_signatures_cover_header():
    assert set(_lib.header_symbols()) <= set(_lib.SIGNATURES)


def test_version_and_components():
    lib = _lib.load()
    assert b"sm_100a" in lib.sky_version()
    assert [lib.sky_theory_components(t) for t in range(6)] == [4, 5, 5, 13, 4, 4]
    assert lib.sky_theory_components(17) == -1
    assert lib.sky_reduce_scratch_size(10) > 0


def _pi(X=8, Y=8, Z=8, C=4, halo=2):
    return np.array([X, Y, Z, halo, 3, C, X * Y * Z, C * X * Y * Z, 1, 1, 1], dtype=np.int32)


def test_invalid_arguments_rejected_before_launch():
    lib = _lib.load()
    pf = np.array([1, 1, 1, 0.2, 0.2, 0.2, 0.008, 0.1, 1.0, 1.0], dtype=np.float64)
    dummy = ctypes.c_void_p(16)
    # unknown theory
    assert lib.sky_gradient_step(9, _lib.i32p(_pi()), 11, _lib.f64p(pf), 10, dummy, dummy, dummy, None) == 1
    # component count does not match the theory
    assert lib.sky_gradient_step(1, _lib.i32p(_pi(C=4)), 11, _lib.f64p(pf), 10, dummy, dummy, dummy, None) == 1
    # halo below the stencil radius
    assert lib.sky_gradient_step(0, _lib.i32p(_pi(halo=1)), 11, _lib.f64p(pf), 10, dummy, dummy, dummy, None) == 1
    # inconsistent dim_grid
    bad = _pi()
    bad[6] += 1
    assert lib.sky_gradient_step(0, _lib.i32p(bad), 11, _lib.f64p(pf), 10, dummy, dummy, dummy, None) == 1
    assert b"dim_grid" in lib.sky_last_error()
    # null buffers
    assert lib.sky_gradient_step(0, _lib.i32p(_pi()), 11, _lib.f64p(pf), 10, None, dummy, dummy, None) == 1
    # scratch too small
    out = ctypes.c_double()
    assert lib.sky_sum(dummy, 10, dummy, 4, ctypes.byref(out), None, None) == 5


def test_init_field_rejects_bad_soliton_lists():
    lib = _lib.load()
    pf = np.array([1, 1, 1, 0.2, 0.2, 0.2, 0.008, 0.1, 1.0, 1.0], dtype=np.float64)
    dummy = ctypes.c_void_p(16)
    b = np.ones(64, np.int32)
    c = np.zeros(3 * 64)
    q = np.tile([1.0, 0.0, 0.0, 0.0], 64)
    args = (_lib.i32p(_pi()), 11, _lib.f64p(pf), 10)
    assert lib.sky_init_field(*args, 49, _lib.i32p(b), _lib.f64p(c), _lib.f64p(q), 1.5, 0, dummy, None) == 1
    b3 = b.copy()
    b3[0] = 3                                         # no B = 3 rational map
    assert lib.sky_init_field(*args, 1, _lib.i32p(b3), _lib.f64p(c), _lib.f64p(q), 1.5, 0, dummy, None) == 1
    assert lib.sky_init_field(*args, 1, _lib.i32p(b), _lib.f64p(c), _lib.f64p(q), 0.0, 0, dummy, None) == 1
    assert lib.sky_init_field(*args, 1, _lib.i32p(b), _lib.f64p(c), _lib.f64p(q), 1.5, 0, None, None) == 1


def test_min_and_arresting_criteria_reject_bad_arguments():
    lib = _lib.load()
    dummy = ctypes.c_void_p(16)
    out = ctypes.c_double()
    assert lib.sky_min(None, 10, dummy, 1 << 20, ctypes.byref(out), None, None) == 1
    assert lib.sky_min(dummy, 10, dummy, 4, ctypes.byref(out), None, None) == 5
    n = lib.sky_reduce_scratch_size(0)
    assert lib.sky_arresting_criteria(_lib.i32p(_pi()), 11, None, dummy, None, dummy, n, ctypes.byref(out), None) == 1
    assert lib.sky_arresting_criteria(_lib.i32p(_pi()), 11, dummy, dummy, None, dummy, 4, ctypes.byref(out), None) == 5
