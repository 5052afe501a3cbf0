"""The `.dat` writer is byte-for-byte the reference's: digests of the reference's own output
for the golden fields (tests/golden/dat_sha256.json, made by make_golden_dat.py) against the
files skyrmion_solver_b200.core.io writes for the same arrays (CPU only)."""
import hashlib
import json
import os

import numpy as np
import pytest

from tests.golden.make_golden_dat import DIRS, bundle_inputs

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("short", list(DIRS))
@pytest.mark.parametrize("precision", [32, 16])
def test_output_bundle_matches_the_reference_bytes(tmp_path, short, precision):
    from skyrmion_solver_b200 import theories as T
    want = json.load(open(os.path.join(HERE, "golden", "dat_sha256.json")))[f"{short}/{precision}"]
    d = dict(np.load(os.path.join(HERE, "golden", f"{short}.npz")))
    T.by_short_name(short).io.output_data_bundle(output_dir=str(tmp_path), precision=precision, **bundle_inputs(d))
    got = {n: hashlib.sha256(open(os.path.join(tmp_path, n), "rb").read()).hexdigest()
           for n in sorted(os.listdir(tmp_path))}
    assert got == want


@pytest.mark.gpu
def test_simulation_save_output(tmp_path):
    """Simulation.save_output writes the bundle from the device state: the field file is the
    writer's bytes for the field, and the densities (computed on the device) read back to the
    reference's golden densities."""
    from skyrmion_solver_b200.core.io import output_field_dat
    from tests import _golden as G
    from tests._gpu import golden_simulation
    d = G.load("omega")
    th, sim = golden_simulation("omega", d)
    X, Y, Z = (int(v) for v in d["p_i"][:3])
    sim.initialize({"mode": "ground"})          # the reference grid (r = h * index)
    from tests._gpu import dev
    sim.Field.copy_(dev(d["field0"]))
    sim.save_output(str(tmp_path / "out"), precision=17)
    output_field_dat(d["field0"].ravel(), str(tmp_path / "ref.dat"), X, Y, Z, 5, precision=17)
    assert open(tmp_path / "out" / "Field.dat", "rb").read() == open(tmp_path / "ref.dat", "rb").read()
    for name, key in (("EnergyDensity.dat", "energy_density0"), ("BaryonDensity.dat", "baryon_density0")):
        vals = np.array(open(tmp_path / "out" / name).read().split(), dtype=np.float64)
        ref = d[key].ravel()
        assert vals.shape == ref.shape
        assert np.max(np.abs(vals - ref)) <= 1e-12 * max(1.0, float(np.max(np.abs(ref))))
    assert (tmp_path / "out" / "OmegaMeson.dat").exists() and (tmp_path / "out" / "xGrid.dat").exists()
