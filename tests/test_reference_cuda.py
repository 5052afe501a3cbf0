"""The reference's own code on the GPU (Numba-CUDA), from the copy installed under baseline/_ref.

1. Drop-in: the reference's unmodified ``Simulation`` class (core/simulation.py) built with this
   package's theory module (params, kernels, observables).  Its ``step`` runs the reference's own
   ``do_arrested_newton_flow`` (core/integrator.py:284-410), its own Numba RK4 stage and finalize
   kernels and its own max reduction, and calls this package's gradient launchable and energy
   observable on Numba device arrays.  Three steps from the golden inputs match the golden steps
   that the reference produced (1e-10 relative per step, as the other step parity tests).
2. The reference's own theory kernels (its Numba gradient, energy and norm kernels) and this
   package's drop-in path agree step by step from the same field (1e-10 relative energy), on a
   ragged 40 x 36 x 44 lattice and at the full sizes of two benchmark configurations: the
   nuclear 64^3 seeded hedgehog (h = 0.2) and the omega B = 4 rational map on 128^3 (h = 0.15).

Skipped when the reference is not installed (``tests/_reference.py`` says how to install it).
"""
import numpy as np
import pytest

from tests import _golden as G
from tests import _reference as R

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not R.available(), reason="the reference is not installed under baseline/_ref")]

STEP_TOL = 1e-10


@pytest.mark.parametrize("name", ["nuclear", "omega", "rho"])
def test_reference_simulation_drives_this_packages_theory(name):
    from skyrmion_solver_b200 import theories as T
    from tests.golden.make_golden import theory_params
    _, Simulation, _ = R.load(())
    th = T.by_short_name(name)
    d = G.load(name)
    sim = Simulation(theory_params(name, th).resolved(), th)      # the reference's own class
    assert np.array_equal(sim.p_i_h, d["p_i"]) and np.array_equal(sim.p_f_h, d["p_f"])
    shp = d["field0"].shape
    sim.Field.copy_to_device(np.ascontiguousarray(d["field0"].ravel()))
    sim.Velocity.copy_to_device(np.ascontiguousarray(d["velocity0"].ravel()))
    for s in range(len(d["energies"])):
        E, err = sim.step(float(d[f"prev{s}"]))
        assert abs(E - d["energies"][s]) <= STEP_TOL * abs(d["energies"][s]), (s, E, d["energies"][s])
        assert abs(err - d["errs"][s]) <= STEP_TOL * abs(d["errs"][s])
        assert G.rel_err(sim.Field.copy_to_host().reshape(shp), d[f"field{s + 1}"]) <= STEP_TOL
        v = sim.Velocity.copy_to_host().reshape(shp)
        if np.any(d[f"velocity{s + 1}"]):
            assert G.rel_err(v, d[f"velocity{s + 1}"]) <= STEP_TOL
        else:
            assert not np.any(v)


@pytest.mark.parametrize("name", ["omega"])
def test_reference_kernels_and_drop_in_agree(name):
    """The reference's own theory on a 40 x 36 x 44 lattice with seeded off-sphere inputs against
    this package's Simulation (the same reference layout, FP64), three steps."""
    import torch
    from skyrmion_solver_b200 import theories as T
    from skyrmion_solver_b200.core.simulation import Simulation as OurSimulation
    from tests.test_march import inputs
    theories, Simulation, _ = R.load((name,))
    ref_th = theories[name]
    dims, h = (40, 36, 44), (0.2, 0.2, 0.2)
    kw = dict(xlen=dims[0], ylen=dims[1], zlen=dims[2], lsx=h[0], lsy=h[1], lsz=h[2], xsize=h[0] * (dims[0] - 1),
              ysize=h[1] * (dims[1] - 1), zsize=h[2] * (dims[2] - 1), time_step=0.04)
    ref = Simulation(ref_th.params.Params(**kw), ref_th)
    ours = OurSimulation(T.by_short_name(name).params.default_params(**kw), T.by_short_name(name))
    assert np.array_equal(ref.p_i_h, ours.p_i_h) and np.array_equal(ref.p_f_h, ours.p_f_h)
    F, V = inputs(int(ref.p_i_h[5]), dims, h=h, seed=11)
    ref.Field.copy_to_device(np.ascontiguousarray(F.ravel()))
    ref.Velocity.copy_to_device(np.ascontiguousarray(V.ravel()))
    ours.Field.copy_(torch.from_numpy(F.ravel()))
    ours.Velocity.copy_(torch.from_numpy(V.ravel()))
    er = ref.observables()["energy"]
    eo = ours.observables()["energy"]
    assert abs(er - eo) <= STEP_TOL * abs(er)
    for s in range(3):
        er, errr = ref.step(er)
        eo, erro = ours.step(eo)
        assert abs(er - eo) <= STEP_TOL * abs(er), (s, er, eo)
        assert abs(errr - erro) <= STEP_TOL * max(1.0, abs(errr)), (s, errr, erro)
    fr = ref.Field.copy_to_host()
    fo = ours.Field.cpu().numpy()
    assert G.rel_err(fo, fr) <= STEP_TOL


def _configured(name):
    from tests.test_config_parity import _nuclear64, _omega128
    return {"nuclear64": _nuclear64, "omega128": _omega128}[name]()


@pytest.mark.parametrize("key", ["nuclear64", "omega128"])
def test_reference_kernels_and_drop_in_agree_at_config_size(key):
    """The reference's Simulation with its own theory module against this package's Simulation on a
    benchmark configuration's full lattice, from the field this package's initialiser builds (the
    seeded hedgehog with noise, or the B = 4 rational map with omega seeded as -c_omega B0): two
    FP64 arrested-Newton steps, energy, err and field within 1e-10 relative."""
    import torch
    from skyrmion_solver_b200.core.simulation import Simulation as OurSimulation
    th, p, cfg = _configured(key)
    theories, Simulation, _ = R.load((th.SHORT_NAME,))
    ref_th = theories[th.SHORT_NAME]
    ours = OurSimulation(p, th)
    ours.initialize(cfg)
    torch.cuda.synchronize()
    kw = {k: getattr(p, k) for k in ("xlen", "ylen", "zlen", "lsx", "lsy", "lsz", "xsize", "ysize", "zsize",
                                     "time_step", "killkinen")}
    ref = Simulation(ref_th.params.Params(**kw), ref_th)
    assert np.array_equal(ref.p_i_h, ours.p_i_h) and np.array_equal(ref.p_f_h, ours.p_f_h)
    ref.Field.copy_to_device(np.ascontiguousarray(ours.Field.cpu().numpy()))
    ref.Velocity.copy_to_device(np.zeros(ours.Velocity.numel()))
    er = ref.observables()["energy"]
    eo = ours.observables()["energy"]
    assert abs(er - eo) <= STEP_TOL * abs(er)
    for s in range(2):
        er, errr = ref.step(er)
        eo, erro = ours.step(eo)
        assert abs(er - eo) <= STEP_TOL * abs(er), (s, er, eo)
        assert abs(errr - erro) <= STEP_TOL * max(1.0, abs(errr)), (s, errr, erro)
    assert G.rel_err(ours.Field.cpu().numpy(), ref.Field.copy_to_host()) <= STEP_TOL


def test_config1_time_step_diverges_in_the_reference_too():
    """The nuclear 64^3 configuration's dt = 0.5 h is beyond RK4's stability limit for the
    reference's own code: its unmodified Simulation (Numba-CUDA kernels) and this package's
    drop-in path both blow up, at the same step, from the same seeded field."""
    import math
    import torch
    from skyrmion_solver_b200.core.simulation import Simulation as OurSimulation
    th, p, cfg = _configured("nuclear64")
    theories, Simulation, _ = R.load(("nuclear",))
    ours = OurSimulation(p, th)
    ours.initialize(cfg)
    torch.cuda.synchronize()
    kw = {k: getattr(p, k) for k in ("xlen", "ylen", "zlen", "lsx", "lsy", "lsz", "xsize", "ysize", "zsize",
                                     "time_step", "killkinen")}
    ref = Simulation(theories["nuclear"].params.Params(**kw), theories["nuclear"])
    ref.Field.copy_to_device(np.ascontiguousarray(ours.Field.cpu().numpy()))
    ref.Velocity.copy_to_device(np.zeros(ours.Velocity.numel()))
    er, eo = ref.observables()["energy"], ours.observables()["energy"]
    first = {}
    for n in range(1, 121):
        if "ref" not in first:
            er, _ = ref.step(er)
            if not math.isfinite(er):
                first["ref"] = n
        if "ours" not in first:
            eo, _ = ours.step(eo)
            if not math.isfinite(eo):
                first["ours"] = n
        if len(first) == 2:
            break
    assert len(first) == 2 and first["ref"] == first["ours"], first
