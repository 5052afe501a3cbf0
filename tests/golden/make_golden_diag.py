"""Golden values of the reference's nuclear-model diagnostics, produced by the
reference itself under Numba's CUDA simulator (the same harness as
make_golden.py: `python tests/golden/make_golden_diag.py`, after make_golden.py).

On the golden field `field0` of nuclear.npz it records the reference's
Simulation.compute_center_of_mass, compute_rms_radius, compute_U_tensor,
compute_V_tensor, compute_W_tensor, compute_quadrupole_tensor and
compute_D_term (core/simulation.py:390-500, th/nuclear_skyrme/observables.py:
182-487) into nuclear_diag.npz.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from tests.golden.make_golden import load_reference, theory_params  # noqa: E402


def main():
    theories, Simulation = load_reference()
    th = theories["nuclear"]
    sim = Simulation(theory_params("nuclear", th), th)
    sim.initialize({"mode": "ground"})
    d = dict(np.load(os.path.join(HERE, "nuclear.npz")))
    assert np.array_equal(np.asarray(sim.p_i_h), d["p_i"]) and np.array_equal(np.asarray(sim.p_f_h), d["p_f"])
    sim.Field.copy_to_device(d["field0"].ravel())
    out = dict(p_i=d["p_i"], p_f=d["p_f"], field=d["field0"])
    out["com"] = np.asarray(sim.compute_center_of_mass(), dtype=np.float64)
    out["rms"] = np.float64(sim.compute_rms_radius())
    out["U"] = np.asarray(sim.compute_U_tensor(), dtype=np.float64)
    out["V"] = np.asarray(sim.compute_V_tensor(), dtype=np.float64)
    out["W"] = np.asarray(sim.compute_W_tensor(), dtype=np.float64)
    out["Q"] = np.asarray(sim.compute_quadrupole_tensor(), dtype=np.float64)
    out["D"] = np.float64(sim.compute_D_term())
    path = os.path.join(HERE, "nuclear_diag.npz")
    np.savez_compressed(path, **out)
    print({k: v for k, v in out.items() if k not in ("field", "p_i", "p_f")}, flush=True)
    print(f"wrote {path}", flush=True)


if __name__ == "__main__":
    main()
