"""Marching x-plane kernels on ragged geometries, against the FP64 oracle.

The marching kernels split a lattice into (x-chunk, 8-row y, 32-column z) tiles
and stream x-planes through a five-slot shared-memory ring; these tests use
grid sizes that are not multiples of the tile, several x-chunk lengths
(including chunks of 4 planes, so most sites sit next to a chunk seam) and the
3-D tile kernels as a second opinion.  Tolerances: 1e-12 relative per gradient
evaluation, 1e-10 relative per arrested-Newton step (FP64).
"""
import numpy as np
import pytest

from oracle import skyrme_oracle as O
from tests import _golden as G

pytestmark = pytest.mark.gpu

GRAD_TOL = 1e-12
STEP_TOL = 1e-10

EXTRA = {
    "nuclear": dict(mpi=0.8, kappa=1.3),
    "omega": dict(),
    "coulomb": dict(),
    "rho": dict(mpi=0.586, mrho=3.29, c_alpha=0.2256, time_step=0.01),
    "berger": dict(mpi=0.9, kappa=1.1, alpha=1.3),
    "lightly_bound": dict(mpi=0.7, alpha=0.3),
}


def params_for(short, dims, h=(0.2, 0.18, 0.22)):
    from skyrmion_solver_b200 import theories as T
    th = T.by_short_name(short)
    kw = dict(xlen=dims[0], ylen=dims[1], zlen=dims[2], lsx=h[0], lsy=h[1], lsz=h[2],
              xsize=h[0] * (dims[0] - 1), ysize=h[1] * (dims[1] - 1), zsize=h[2] * (dims[2] - 1),
              time_step=0.02, killkinen=True, newtonflow=True, unit_length=True)
    kw.update(EXTRA[short])
    p = th.params.default_params(**kw)
    p_i, p_f = th.params.pack_device_params(p.resolved())
    return th, np.asarray(p_i, np.int32), np.asarray(p_f, np.float64)


def inputs(C, dims, h=(0.2, 0.18, 0.22), seed=0):
    rng = np.random.default_rng(seed)
    X, Y, Z = dims
    xs = (np.arange(X) - (X - 1) / 2.0) * h[0]
    ys = (np.arange(Y) - (Y - 1) / 2.0) * h[1]
    zs = (np.arange(Z) - (Z - 1) / 2.0) * h[2]
    x, y, z = np.meshgrid(xs, ys, zs, indexing="ij")
    r = np.sqrt(x * x + y * y + z * z)
    f = np.pi * np.exp(-r / 1.1)
    rs = np.where(r > 0, r, 1.0)
    F = np.zeros((C,) + tuple(dims))
    F[0] = np.cos(f)
    F[1], F[2], F[3] = np.sin(f) * x / rs, np.sin(f) * y / rs, np.sin(f) * z / rs
    F[:4] += rng.uniform(-0.02, 0.02, size=(4,) + tuple(dims))
    F[:4] /= np.sqrt((F[:4] ** 2).sum(axis=0))
    for a in range(4, C):
        F[a] = 0.3 * np.exp(-r * r / 2) * np.cos((a - 3) * x + 0.5 * y) + rng.uniform(-0.01, 0.01, size=dims)
    V = rng.uniform(-1e-2, 1e-2, size=F.shape)
    return F, V


def _set_option(key, value):
    from skyrmion_solver_b200 import _lib
    _lib.call("sky_set_option", key, value)


@pytest.fixture
def options():
    from skyrmion_solver_b200 import _lib
    lib = _lib.load()
    saved = (lib.sky_get_option(0), lib.sky_get_option(1))
    yield
    _set_option(0, saved[0])
    _set_option(1, saved[1])


def _plain_gradient(name, F, p_i, p_f):
    import torch
    from skyrmion_solver_b200 import _lib
    from skyrmion_solver_b200._lib import THEORY_IDS, f64p, i32p
    t = torch.from_numpy(F.ravel().copy()).cuda()
    eg = torch.zeros_like(t)
    l = torch.zeros_like(t)
    _lib.call("sky_gradient_step", THEORY_IDS[name], i32p(p_i), len(p_i), f64p(p_f), len(p_f), _lib.dptr(l),
              _lib.dptr(t), _lib.dptr(eg), _lib.stream_ptr())
    torch.cuda.synchronize()
    return eg.cpu().numpy().reshape(F.shape), l.cpu().numpy().reshape(F.shape)


@pytest.mark.parametrize("name", ["nuclear", "omega", "coulomb", "rho", "berger", "lightly_bound"])
@pytest.mark.parametrize("dims", [(37, 21, 70), (9, 33, 5), (6, 6, 40)])
def test_plain_gradient_geometry(options, name, dims):
    th, p_i, p_f = params_for(name, dims)
    C = int(p_i[5])
    F, _ = inputs(C, dims, seed=sum(dims))
    ref_eg, ref_l = O.gradient(O.THEORIES[name], F, p_i, p_f)
    _set_option(0, 0)
    tile_eg, _ = _plain_gradient(name, F, p_i, p_f)
    assert G.rel_err(tile_eg, ref_eg) <= GRAD_TOL
    _set_option(0, 1)
    for xc in (0, 4, 7):
        _set_option(1, xc)
        eg, l = _plain_gradient(name, F, p_i, p_f)
        assert G.rel_err(eg, ref_eg) <= GRAD_TOL, (xc, G.rel_err(eg, ref_eg))
        assert G.rel_err(l, ref_l) <= GRAD_TOL


@pytest.mark.parametrize("name", ["nuclear", "omega", "coulomb", "rho"])
def test_engine_fp64_chunked(name):
    from skyrmion_solver_b200.engine import Engine
    dims = (29, 19, 45)
    th, p_i, p_f = params_for(name, dims)
    C = int(p_i[5])
    F, V = inputs(C, dims, seed=3)
    thd = O.THEORIES[name]
    E = O.total_energy(thd, F, p_i, p_f)
    Fr, Vr = F, V
    ref = []
    for _ in range(2):
        Fr, Vr, E, err, _ = O.arrested_newton_step(thd, Fr, Vr, p_i, p_f, E)
        ref.append((Fr, Vr, E, err))
    with Engine(0) as eng:
        iid = eng.add(name, (p_i, p_f), F, V, precision="fp64")
        eng.retile(iid, 5)
        assert eng.xc(iid) == 5
        for n in range(2):
            eng.step(1)
            st = eng.stats(iid)
            assert abs(st.energy - ref[n][2]) <= STEP_TOL * abs(ref[n][2])
            assert abs(st.err - ref[n][3]) <= STEP_TOL * max(1.0, abs(ref[n][3]))
        f, v = eng.read(iid)
        assert G.rel_err(f, ref[1][0]) <= STEP_TOL
        if np.any(ref[1][1]):
            assert G.rel_err(v, ref[1][1]) <= STEP_TOL


@pytest.mark.parametrize("xc", [0, 4])
def test_engine_rho_fp32_marching(xc):
    """rho (13 components) marches in FP32 without register queues (mixed x-derivatives
    from taps across the ring planes): two steps against the FP64 oracle, FP32 tolerance."""
    from skyrmion_solver_b200.engine import Engine
    dims = (29, 19, 45)
    th, p_i, p_f = params_for("rho", dims)
    F, V = inputs(13, dims, seed=7)
    thd = O.THEORIES["rho"]
    Fr, Vr, E = F, V, O.total_energy(thd, F, p_i, p_f)
    ref = []
    for _ in range(2):
        Fr, Vr, E, err, _ = O.arrested_newton_step(thd, Fr, Vr, p_i, p_f, E)
        ref.append((Fr, E))
    with Engine(0) as eng:
        iid = eng.add("rho", (p_i, p_f), F, V, precision="fp32")
        if xc:
            eng.retile(iid, xc)
            assert eng.xc(iid) == xc
        assert eng.xc(iid) > 0
        for n in range(2):
            eng.step(1)
            st = eng.stats(iid)
            assert abs(st.energy - ref[n][1]) <= 2e-5 * abs(ref[n][1]), (n, st.energy, ref[n][1])
        f, _ = eng.read(iid)
    assert G.rel_err(f, ref[1][0]) <= 2e-5


@pytest.mark.parametrize("name", ["omega", "rho"])
def test_engine_fp32_tiling_invariance(name):
    """Re-tiling changes only the order of the per-tile energy partials: the trajectory is unchanged."""
    from skyrmion_solver_b200.engine import Engine
    dims = (40, 24, 36)
    th, p_i, p_f = params_for(name, dims)
    F, V = inputs(int(p_i[5]), dims, seed=5)
    with Engine(0) as a, Engine(0) as b:
        ia = a.add(name, (p_i, p_f), F, V, precision="fp32")
        ib = b.add(name, (p_i, p_f), F, V, precision="fp32")
        b.retile(ib, 4)
        a.step(6)
        b.step(6)
        fa, _ = a.read(ia)
        fb, _ = b.read(ib)
        assert np.array_equal(fa, fb)
        assert a.stats(ia).energy == pytest.approx(b.stats(ib).energy, rel=1e-13)


def _plain_density(name, F, p_i, p_f, fn):
    import ctypes
    import torch
    from skyrmion_solver_b200 import _lib
    from skyrmion_solver_b200._lib import THEORY_IDS, f64p, i32p
    from skyrmion_solver_b200.core.utils import scratch_doubles
    t = torch.from_numpy(F.ravel().copy()).cuda()
    en = torch.zeros(int(p_i[6]), dtype=torch.float64, device="cuda")
    _lib.call(fn, THEORY_IDS[name], i32p(p_i), len(p_i), f64p(p_f), len(p_f), _lib.dptr(en), _lib.dptr(t),
              _lib.stream_ptr())
    scratch = torch.zeros(scratch_doubles(), dtype=torch.float64, device="cuda")
    tot = ctypes.c_double()
    _lib.call(fn.replace("_density", "").replace("sky_energy", "sky_total_energy").replace("sky_baryon",
                                                                                          "sky_total_baryon"),
              THEORY_IDS[name], i32p(p_i), len(p_i), f64p(p_f), len(p_f), _lib.dptr(t), _lib.dptr(scratch),
              scratch.numel(), ctypes.byref(tot), _lib.stream_ptr())
    torch.cuda.synchronize()
    return en.cpu().numpy().reshape(F.shape[1:]), tot.value


@pytest.mark.parametrize("name", ["nuclear", "omega", "coulomb", "rho", "berger"])
@pytest.mark.parametrize("dims", [(37, 21, 70), (9, 33, 5)])
def test_plain_density_geometry(options, name, dims):
    th, p_i, p_f = params_for(name, dims)
    F, _ = inputs(int(p_i[5]), dims, seed=sum(dims) + 1)
    thd = O.THEORIES[name]
    for mode in (1, 0):
        _set_option(0, mode)
        e, E = _plain_density(name, F, p_i, p_f, "sky_energy_density")
        b, Bn = _plain_density(name, F, p_i, p_f, "sky_baryon_density")
        ref_e = O.energy_density(thd, F, p_i, p_f)
        ref_b = O.baryon_density(thd, F, p_i, p_f)
        assert G.rel_err(e, ref_e) <= GRAD_TOL and G.rel_err(b, ref_b) <= GRAD_TOL
        assert abs(E - O.total_energy(thd, F, p_i, p_f)) <= 1e-12 * abs(E)
        assert abs(Bn - O.total_baryon(thd, F, p_i, p_f)) <= 1e-12 * max(1.0, abs(Bn))
