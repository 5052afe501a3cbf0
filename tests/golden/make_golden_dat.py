"""SHA-256 digests of the reference's own `.dat` output for the golden fields
(`python tests/golden/make_golden_dat.py`, reading the reference from /root/reference).

For every theory, the reference's theory io module (th/*/io.py over core/io.py)
writes its output bundle for the golden field `field0`, the reference grid
(r = h * index) and the golden energy / baryon densities, at precision 32 and
16; the digest of every file goes to dat_sha256.json.  tests/test_io.py writes
the same bundles with skyrmion_solver_b200.core.io and compares the digests.
"""
import hashlib
import importlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REFERENCE_ROOT = os.environ.get("SKY_REFERENCE_ROOT", "/root/reference")
DIRS = {"nuclear": "nuclear_skyrme", "omega": "omega_skyrme", "coulomb": "coulomb_skyrme", "rho": "rho_skyrme",
        "berger": "berger_skyrme", "lightly_bound": "lightly_bound_skyrme"}


def bundle_inputs(d):
    p_i, p_f = d["p_i"], d["p_f"]
    X, Y, Z = (int(v) for v in p_i[:3])
    grid = np.stack(np.meshgrid(p_f[3] * np.arange(X), p_f[4] * np.arange(Y), p_f[5] * np.arange(Z),
                                indexing="ij")).ravel()
    return dict(h_Field=d["field0"].ravel(), h_EnergyDensity=d["energy_density0"].ravel(),
                h_BaryonDensity=d["baryon_density0"].ravel(), h_grid=grid, xlen=X, ylen=Y, zlen=Z,
                number_coordinates=int(p_i[4]), number_total_fields=int(p_i[5]))


def digests(folder):
    out = {}
    for name in sorted(os.listdir(folder)):
        with open(os.path.join(folder, name), "rb") as fh:
            out[name] = hashlib.sha256(fh.read()).hexdigest()
    return out


def load_io(d_name):
    """The reference theory's io module alone (its package __init__ imports the GL viewer)."""
    import types
    th_dir = os.path.join(REFERENCE_ROOT, "skyrmion_solver", "theories")
    if "skyrmion_solver.theories" not in sys.modules:
        importlib.import_module("skyrmion_solver")
        pkg = types.ModuleType("skyrmion_solver.theories")
        pkg.__path__ = [th_dir]
        sys.modules["skyrmion_solver.theories"] = pkg
    name = "skyrmion_solver.theories." + d_name
    if name not in sys.modules:
        sub = types.ModuleType(name)
        sub.__path__ = [os.path.join(th_dir, d_name)]
        sys.modules[name] = sub
    return importlib.import_module(name + ".io")


def main():
    sys.path.insert(0, REFERENCE_ROOT)
    result = {}
    for short, d_name in DIRS.items():
        io = load_io(d_name)
        d = dict(np.load(os.path.join(HERE, f"{short}.npz")))
        for prec in (32, 16):
            with tempfile.TemporaryDirectory() as tmp:
                io.output_data_bundle(output_dir=tmp, precision=prec, **bundle_inputs(d))
                result[f"{short}/{prec}"] = digests(tmp)
    with open(os.path.join(HERE, "dat_sha256.json"), "w") as fh:
        json.dump(result, fh, indent=1, sort_keys=True)
    print("wrote", os.path.join(HERE, "dat_sha256.json"), sum(len(v) for v in result.values()), "digests")


if __name__ == "__main__":
    main()
