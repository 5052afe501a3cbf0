"""Parity at the benchmark configurations' full sizes.

The reference-produced goldens are 12 x 11 x 10 lattices; these tests run the
device paths on the full lattices of two benchmark configurations and compare
them with the FP64 oracle (itself pinned to those goldens):

* nuclear (pion-only) model, 64^3, h = 0.2, dt = 0.5 h, hedgehog
  f(r) = pi exp(-r/1.5) plus seeded U(-1e-3, 1e-3) noise, renormalised, with
  the two-site vacuum shell: three FP64 arrested-Newton steps of the drop-in
  ``Simulation.step`` and of the resident FP64 engine;
* omega-meson variant, 128^3, h = 0.15, dt = 0.2 h, B = 4 cubic rational map
  f(r) = pi exp(-r/2) with omega seeded as -c_omega B0, the parameter class's
  default couplings: two FP64 steps of both paths; with the reference example's
  couplings, sixteen defect-corrected FP32 (``fp32d``) engine steps against
  sixteen FP64 engine steps.

The oracle's arrested-Newton step follows core/integrator.py:284-410 of the
reference.  Tolerances: 1e-10 relative per step for FP64 (energy, err, field,
velocity), 2e-5 relative for fp32d against FP64 after sixteen steps.
"""
import numpy as np
import pytest

from oracle import skyrme_oracle as O
from tests import _golden as G

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-10
FP32D_TOL = 2e-5


def _nuclear64():
    from skyrmion_solver_b200 import theories as T
    th = T.by_short_name("nuclear")
    h, L = 0.2, 64
    p = th.params.default_params(xlen=L, ylen=L, zlen=L, lsx=h, lsy=h, lsz=h, xsize=h * (L - 1),
                                 ysize=h * (L - 1), zsize=h * (L - 1), time_step=0.5 * h, killkinen=True)
    cfg = {"mode": "hedgehog", "scale": 1.5, "noise": 1e-3, "seed": 0, "vacuum_shell": 2}
    return th, p, cfg


# couplings of the reference's omega example (examples/omega_skyrme_gl.py:12-15), on which the
# relaxation is stable; with the parameter class's defaults (c_omega = 34.7) the 128^3 flow
# diverges within sixteen steps in FP64 as well
EXAMPLE_OMEGA = dict(f_pi=139.8, m_pi=43.91, m_omega=249.5, beta_omega=8.036)


def _omega128(**couplings):
    from skyrmion_solver_b200 import theories as T
    th = T.by_short_name("omega")
    h, L = 0.15, 128
    p = th.params.default_params(xlen=L, ylen=L, zlen=L, lsx=h, lsy=h, lsz=h, xsize=h * (L - 1),
                                 ysize=h * (L - 1), zsize=h * (L - 1), time_step=0.2 * h, killkinen=True,
                                 **couplings)
    cfg = {"mode": "rational_map", "baryon_number": 4, "scale": 2.0, "vacuum_shell": 2}
    return th, p, cfg


_CACHE = {}


def _oracle_run(key, nsteps):
    """(p_i, p_f, initial field, [(F, V, E, err) per step]) of the oracle from the field the
    drop-in Simulation initialises (read back from the device, FP64)."""
    if key in _CACHE:
        return _CACHE[key]
    import torch
    from skyrmion_solver_b200.core.simulation import Simulation
    th, p, cfg = {"nuclear64": _nuclear64, "omega128": _omega128,
                  "omega128_example": lambda: _omega128(**EXAMPLE_OMEGA)}[key]()
    sim = Simulation(p, th)
    sim.initialize(cfg)
    torch.cuda.synchronize()
    p_i, p_f = np.asarray(sim.p_i_h, np.int32), np.asarray(sim.p_f_h, np.float64)
    shape = (int(p_i[5]),) + tuple(int(v) for v in p_i[:3])
    F0 = sim.Field.cpu().numpy().reshape(shape).copy()
    V0 = np.zeros_like(F0)
    del sim
    thd = O.THEORIES[th.SHORT_NAME]
    e0 = O.total_energy(thd, F0, p_i, p_f)
    traj = []
    F, V, prev = F0, V0, e0
    for _ in range(nsteps):
        F, V, E, err, _ = O.arrested_newton_step(thd, F, V, p_i, p_f, prev)
        traj.append((F, V, E, err))
        prev = E
    _CACHE[key] = (th, p, cfg, p_i, p_f, F0, e0, traj)
    return _CACHE[key]


def _check_step(n, E, err, F, V, ref):
    Fr, Vr, Er, errr = ref
    assert abs(E - Er) <= FP64_TOL * abs(Er), (n, E, Er)
    assert abs(err - errr) <= FP64_TOL * max(1.0, abs(errr)), (n, err, errr)
    assert G.rel_err(F, Fr) <= FP64_TOL, n
    if np.any(Vr):
        assert G.rel_err(V, Vr) <= FP64_TOL, n
    else:
        assert not np.any(V), n


def _simulation_steps(key, nsteps):
    import torch
    from skyrmion_solver_b200.core.simulation import Simulation
    th, p, cfg, p_i, p_f, F0, e0, traj = _oracle_run(key, nsteps)
    sim = Simulation(p, th)
    sim.initialize(cfg)
    e = sim.observables()["energy"]
    assert abs(e - e0) <= 1e-12 * abs(e0)
    assert np.array_equal(sim.Field.cpu().numpy().reshape(F0.shape), F0)
    for n in range(nsteps):
        E, err = sim.step(e)
        torch.cuda.synchronize()
        F = sim.Field.cpu().numpy().reshape(F0.shape)
        V = sim.Velocity.cpu().numpy().reshape(F0.shape)
        _check_step(n + 1, E, err, F, V, traj[n])
        e = E


def _engine_steps(key, nsteps):
    from skyrmion_solver_b200.engine import Engine
    th, p, cfg, p_i, p_f, F0, e0, traj = _oracle_run(key, nsteps)
    with Engine(0) as eng:
        i = eng.add(th.SHORT_NAME, (p_i, p_f), F0, None, precision="fp64")
        assert abs(eng.stats(i).energy - e0) <= 1e-12 * abs(e0)
        for n in range(nsteps):
            eng.step(1)
            st = eng.stats(i)
            F, V = eng.read(i)
            _check_step(n + 1, st.energy, st.err, F, V, traj[n])


def test_nuclear_64_simulation_steps_match_oracle():
    _simulation_steps("nuclear64", 3)


def test_nuclear_64_engine_fp64_steps_match_oracle():
    _engine_steps("nuclear64", 3)


def test_omega_128_simulation_steps_match_oracle():
    _simulation_steps("omega128", 2)


def test_omega_128_engine_fp64_steps_match_oracle():
    _engine_steps("omega128", 2)


def test_omega_128_fp32d_tracks_fp64():
    """Sixteen defect-corrected FP32 steps (the FP64 correction is refreshed every sixteen
    steps) against sixteen FP64 engine steps from the same field, with the reference example's
    couplings: energy, baryon number and field within 2e-5 relative."""
    from skyrmion_solver_b200.engine import Engine
    th, p, cfg, p_i, p_f, F0, e0, traj = _oracle_run("omega128_example", 0)
    with Engine(0) as eng:
        a = eng.add("omega", (p_i, p_f), F0, None, precision="fp64")
        b = eng.add("omega", (p_i, p_f), F0, None, precision="fp32d")
        eng.step(16)
        sa, sb = eng.stats(a), eng.stats(b)
        fa, _ = eng.read(a, velocity=False)
        fb, _ = eng.read(b, velocity=False)
    assert sb.precision == "fp32d" and sb.step == 16
    assert abs(sb.energy - sa.energy) <= FP32D_TOL * abs(sa.energy), (sb.energy, sa.energy)
    assert abs(sb.baryon - sa.baryon) <= FP32D_TOL * abs(sa.baryon), (sb.baryon, sa.baryon)
    assert G.rel_err(fb, fa) <= FP32D_TOL


def test_served_fp32d_solve_reaches_the_fp64_energy_and_baryon_number():
    """A solve served in the defect-corrected FP32 schedule (then FP64 to max|g| <= 1e-6) ends
    within 1e-6 relative energy and 1e-4 baryon number of the FP64 solve of the same request:
    a nuclear B = 1 hedgehog on 40^3 (h = 0.25), each through the continuous-batching server."""
    from skyrmion_solver_b200 import serving, theories as T
    from skyrmion_solver_b200.engine import Engine
    th = T.by_short_name("nuclear")
    h, L = 0.25, 40
    p = th.params.default_params(xlen=L, ylen=L, zlen=L, lsx=h, lsy=h, lsz=h, xsize=h * (L - 1),
                                 ysize=h * (L - 1), zsize=h * (L - 1), time_step=0.2 * h)
    p_i, p_f = th.params.pack_device_params(p.resolved())
    init = {"mode": "hedgehog", "scale": 1.0, "vacuum_shell": 2}
    res = {}
    for mode in ("fp64", "fp32d"):
        with Engine(0) as eng:
            srv = serving.Server(eng, chunk=256, fp32_mode=mode)
            srv.submit(serving.Request(0, "nuclear", np.asarray(p_i, np.int32), np.asarray(p_f, np.float64),
                                       None, arrival=0.0, tol=1e-6, max_steps=200_000, init=init))
            out = srv.run()
        assert len(out) == 1 and out[0].status == "converged", (mode, out)
        res[mode] = out[0]
    a, b = res["fp64"], res["fp32d"]
    assert abs(b.energy - a.energy) <= 1e-6 * abs(a.energy), (b.energy, a.energy)
    assert abs(b.baryon - a.baryon) <= 1e-4, (b.baryon, a.baryon)
    assert b.fp32_steps > 0
