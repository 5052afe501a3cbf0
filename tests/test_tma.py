"""TMA plane staging of the engine's stage kernels against cp.async staging.

The stage kernels stage each haloed x-plane either by per-thread cp.async
copies or by one tensor-memory-accelerator box copy per source (library option
2).  Both feed the same ring and the same arithmetic in the same order, so an
instance stepped with either staging must give bitwise identical statistics
and fields.  Lattices here have Z a multiple of 4 (the FP32 TMA row-pitch rule)
but ragged X, Y and Z against the 8 x 32 (y, z) tiles, so boxes cross every
lattice face; velocities start non-zero, and the arrest zeroes them on later
steps (the velocity source is then not copied at all).  The FP64 instances are
also checked against the oracle (1e-10 relative per step).
"""
import numpy as np
import pytest

from oracle import skyrme_oracle as O
from tests import _golden as G
from tests.test_march import inputs, params_for

pytestmark = pytest.mark.gpu


def _run(name, dims, precision, staging, nsteps, seed=5):
    from skyrmion_solver_b200 import _lib
    from skyrmion_solver_b200.engine import Engine
    th, p_i, p_f = params_for(name, dims)
    F, V = inputs(int(p_i[5]), dims, seed=seed)
    old = int(_lib.load().sky_get_option(2))
    old_pair = int(_lib.load().sky_get_option(3))
    _lib.call("sky_set_option", 2, 1 if staging == "tma" else 0)
    _lib.call("sky_set_option", 3, 0)   # one site per thread in both stagings (z-pairs: below)
    try:
        with Engine(0) as eng:
            i = eng.add(name, (p_i, p_f), F, V, precision=precision)
            recs = []
            for _ in range(nsteps):
                eng.step(1)
                s = eng.stats(i)
                recs.append((s.energy, s.baryon, s.err, s.gabs, s.arrested, s.kinetic))
            f, v = eng.read(i)
    finally:
        _lib.call("sky_set_option", 2, old)
        _lib.call("sky_set_option", 3, old_pair)
    return recs, f, v, (F, V, p_i, p_f)


@pytest.mark.parametrize("name,precision", [("omega", "fp32d"), ("omega", "fp32"), ("nuclear", "fp32c"),
                                            ("coulomb", "fp32"), ("berger", "fp32d"), ("rho", "fp32"), ("rho", "fp32d"),
                                            ("omega", "fp64"), ("nuclear", "fp64")])
def test_tma_staging_equals_cp_async_staging(name, precision):
    dims = (23, 13, 44)
    a = _run(name, dims, precision, "tma", 6)
    b = _run(name, dims, precision, "cp.async", 6)
    assert a[0] == b[0]
    assert np.array_equal(a[1], b[1]) and np.array_equal(a[2], b[2])


@pytest.mark.parametrize("name", ["omega", "lightly_bound"])
def test_tma_fp64_engine_matches_oracle(name):
    dims = (19, 11, 36)
    nsteps = 3
    recs, f, v, (F, V, p_i, p_f) = _run(name, dims, "fp64", "tma", nsteps)
    th = O.THEORIES[name]
    E = O.total_energy(th, F, p_i, p_f)
    for n in range(nsteps):
        F, V, E, err, _ = O.arrested_newton_step(th, F, V, p_i, p_f, E)
        assert abs(recs[n][0] - E) <= 1e-10 * abs(E), (n, recs[n][0], E)
        assert abs(recs[n][2] - err) <= 1e-10 * max(1.0, abs(err))
    assert G.rel_err(f, F) <= 1e-10
    if np.any(V):
        assert G.rel_err(v, V) <= 1e-10
    else:
        assert not np.any(v)


def test_tma_option_is_validated():
    from skyrmion_solver_b200 import _lib
    from skyrmion_solver_b200._lib import SkyInvalidArgument
    with pytest.raises(SkyInvalidArgument):
        _lib.call("sky_set_option", 2, 7)


def _run_opts(name, dims, precision, opts, nsteps, seed=5):
    from skyrmion_solver_b200 import _lib
    from skyrmion_solver_b200.engine import Engine
    th, p_i, p_f = params_for(name, dims)
    F, V = inputs(int(p_i[5]), dims, seed=seed)
    lib = _lib.load()
    old = {k: int(lib.sky_get_option(k)) for k in opts}
    for k, v in opts.items():
        _lib.call("sky_set_option", k, v)
    try:
        with Engine(0) as eng:
            i = eng.add(name, (p_i, p_f), F, V, precision=precision)
            recs = []
            for _ in range(nsteps):
                eng.step(1)
                s = eng.stats(i)
                recs.append((s.energy, s.baryon, s.err, s.gabs))
            f, _ = eng.read(i, velocity=False)
    finally:
        for k, v in old.items():
            _lib.call("sky_set_option", k, v)
    return recs, f


@pytest.mark.parametrize("precision", ["fp32", "fp32c", "fp32d"])
def test_z_pair_tiles_track_one_site_tiles(precision):
    """The omega FP32 stages with two z-sites per thread (packed FP32x2 arithmetic, option 3)
    against one site per thread: the same arithmetic up to the compiler's choice of fused
    multiply-adds, so energies, baryon numbers, gradients and fields agree to FP32 accuracy
    (2e-6 relative) after six steps on a lattice ragged against the tiles."""
    dims = (23, 13, 44)
    a, fa = _run_opts("omega", dims, precision, {2: 1, 3: 1}, 6)
    b, fb = _run_opts("omega", dims, precision, {2: 1, 3: 0}, 6)
    for ra, rb in zip(a, b):
        for x, y in zip(ra, rb):
            assert abs(x - y) <= 2e-6 * max(1.0, abs(y)), (ra, rb)
    assert G.rel_err(fa, fb) <= 2e-6


def test_staging_switch_keeps_the_trajectory():
    """sky_engine_set_staging between steps (TMA -> cp.async -> TMA) leaves an instance on the
    trajectory of one that stays on TMA staging, bitwise; invalid stagings are refused."""
    from skyrmion_solver_b200._lib import SkyInvalidArgument
    from skyrmion_solver_b200.engine import Engine
    dims = (23, 13, 44)
    th, p_i, p_f = params_for("omega", dims)
    F, V = inputs(int(p_i[5]), dims, seed=5)
    out = []
    for switch in (False, True):
        with Engine(0) as eng:
            i = eng.add("omega", (p_i, p_f), F, V, precision="fp32d")
            assert eng.staging(i)[0]
            for n in range(6):
                if switch and n in (2, 4):
                    eng.set_staging(i, n == 4)
                eng.step(1)
            out.append((eng.stats(i).energy, eng.stats(i).gabs, eng.read(i)))
            if switch:
                with pytest.raises(SkyInvalidArgument):
                    eng.set_staging(i, False, True)          # z-pairs need TMA
                j = eng.add("nuclear", params_for("nuclear", dims)[1:], F[:4], None, precision="fp32")
                with pytest.raises(SkyInvalidArgument):
                    eng.set_staging(j, True, True)           # z-pairs: omega only
                k = eng.add("omega", params_for("omega", (23, 13, 37))[1:], inputs(5, (23, 13, 37), seed=1)[0],
                            None, precision="fp32")
                with pytest.raises(SkyInvalidArgument):
                    eng.set_staging(k, True)                 # Z * 4 bytes is not a multiple of 16
    (ea, ga, (fa, va)), (eb, gb, (fb, vb)) = out
    assert ea == eb and ga == gb
    assert np.array_equal(fa, fb) and np.array_equal(va, vb)


def test_programmatic_dependent_launch_equals_stream_order():
    """Library option 4 (stage launches with programmatic dependent launch, graph-captured)
    against plain stream order: bitwise identical statistics and fields over twenty steps
    (a defect refresh at step 16, arrests), for FP32 and FP64 instances in one engine."""
    from skyrmion_solver_b200 import _lib
    from skyrmion_solver_b200.engine import Engine
    dims = (23, 13, 44)
    runs = []
    old = int(_lib.load().sky_get_option(4))
    try:
        for pdl in (1, 0):
            _lib.call("sky_set_option", 4, pdl)
            with Engine(0) as eng:
                ids = []
                for name, prec in (("omega", "fp32d"), ("nuclear", "fp64"), ("rho", "fp32")):
                    th, p_i, p_f = params_for(name, dims)
                    F, V = inputs(int(p_i[5]), dims, seed=7)
                    ids.append(eng.add(name, (p_i, p_f), F, V, precision=prec))
                eng.step(13)
                eng.step(7)
                runs.append([(eng.stats(i).energy, eng.stats(i).gabs, eng.read(i, velocity=False)[0]) for i in ids])
    finally:
        _lib.call("sky_set_option", 4, old)
    for a, b in zip(*runs):
        assert a[0] == b[0] and a[1] == b[1] and np.array_equal(a[2], b[2])
    from skyrmion_solver_b200._lib import SkyInvalidArgument
    with pytest.raises(SkyInvalidArgument):
        _lib.call("sky_set_option", 4, 2)
