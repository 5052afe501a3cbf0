"""Golden initial fields of the reference, produced by its own initial-configuration
kernels under Numba's CUDA simulator (the harness of make_golden.py):
`python tests/golden/make_golden_init.py`.

For every theory it runs the reference's Simulation.initialize (core/simulation.py:
124-172) with the theory's own initial_config.initialize (th/<theory>/initial_config.py)
on the golden lattice, for the configurations in CASES: the default ansatz of the
parameters, explicit hedgehogs and rational maps (B = 1..9 and a fall-through B),
seeded smorgasbords, the vacuum, and ansatz flags set through the parameters.  The
fields go to init.npz under "<theory>/<case>", with the parameter arrays and the
configuration as JSON.  Theories can run as parallel processes
(`make_golden_init.py nuclear`, ... write init_<theory>.npz), then
`make_golden_init.py --merge` joins them into init.npz.
"""
import importlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from tests.golden.make_golden import THEORY_DIRS, load_reference, theory_params  # noqa: E402

NUCLEAR_ONLY = [("map_b%d" % b, {}, {"mode": "rational_map", "baryon_number": b, "isospin_rotation": 0.3})
                for b in (1, 2, 4, 5, 6, 7, 8, 9, 12)]
CASES = [
    ("default", {}, {}),
    ("hedgehog_b2", {}, {"ansatz": "hedgehog", "baryon_number": 2, "isospin_rotation": 0.4}),
    ("map_b3", {}, {"mode": "rational_map", "baryon_number": 3, "isospin_rotation": 0.3}),
    ("smorgasbord", {}, {"mode": "smorgasbord", "count": 3, "seed": 5, "lump_baryon": 2, "profile_m0": 0.5,
                         "position_scale": 0.25}),
    ("smorgasbord_default", {"baryon_number": 2.0}, {"mode": "smorgasbord", "seed": 1}),
    ("ground", {}, {"mode": "ground"}),
    ("params_map", {"ansatz": "rational_map", "baryon_number": 4.0, "isospin_rotation": 0.2}, {}),
    ("params_uniform", {"ansatz": "uniform"}, {"mode": "initial"}),
]


def main(argv):
    names = argv or list(THEORY_DIRS)
    theories, Simulation = load_reference()
    out = {}
    for short in names:
        th = theories[short]
        th.initial_config = importlib.import_module(
            "skyrmion_solver.theories.%s.initial_config" % THEORY_DIRS[short])
        cases = CASES + (NUCLEAR_ONLY if short == "nuclear" else [])
        for name, over, cfg in cases:
            sim = Simulation(theory_params(short, th, **over), th)
            sim.initialize(dict(cfg))
            key = "%s/%s" % (short, name)
            out[key + "/field"] = sim.Field.copy_to_host()
            out[key + "/velocity_max"] = np.float64(np.abs(sim.Velocity.copy_to_host()).max())
            out[key + "/p_i"] = np.asarray(sim.p_i_h)
            out[key + "/p_f"] = np.asarray(sim.p_f_h)
            out[key + "/config"] = np.array(json.dumps(cfg))
            print(key, "done", flush=True)
    path = os.path.join(HERE, "init.npz" if not argv else "init_%s.npz" % "_".join(argv))
    np.savez_compressed(path, **out)


def merge():
    out = {}
    parts = [os.path.join(HERE, "init_%s.npz" % t) for t in THEORY_DIRS]
    for path in parts:
        out.update(dict(np.load(path)))
    np.savez_compressed(os.path.join(HERE, "init.npz"), **out)
    for path in parts:
        os.remove(path)


if __name__ == "__main__":
    if sys.argv[1:] == ["--merge"]:
        merge()
    else:
        main(sys.argv[1:])
