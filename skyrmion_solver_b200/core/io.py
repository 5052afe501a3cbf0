"""Plain-text ``.dat`` output in the reference's format (skyrmion_solver core/io.py:20-246).

A field is written component by component, then x by x, with one line per
(x, y) holding the zlen values of that row, each followed by a tab; a blank
line closes every x block and every component.  Numbers use Python's
``{:.<precision>g}`` formatting, so the files are byte-for-byte those the
reference writes for the same arrays (tests/test_io.py checks digests of the
reference's own output).  Rows are formatted and written whole.
"""
from __future__ import annotations

import os

import numpy as np


def _fmt(precision: int):
    return f"{{:.{int(precision)}g}}".format


def _rows(block: np.ndarray, fmt) -> str:
    """Rows of a (ylen, zlen) block, each value followed by a tab, each row by a newline."""
    return "".join("\t".join(map(fmt, row)) + "\t\n" for row in block.tolist())


def output_field_dat(field_flat, path: str, xlen: int, ylen: int, zlen: int, nfields: int,
                     precision: int = 32) -> None:
    """Write components 0..nfields-1 of a flattened field (core/io.py:52-92)."""
    fmt = _fmt(precision)
    n = xlen * ylen * zlen
    f = np.asarray(field_flat, dtype=np.float64).reshape(-1)[: nfields * n].reshape(nfields, xlen, ylen, zlen)
    with open(path, "w", newline="\n") as fh:
        for a in range(nfields):
            for x in range(xlen):
                fh.write(_rows(f[a, x], fmt))
                fh.write("\n")
            fh.write("\n")


def output_iteration_data_dat(values, path: str, precision: int = 32) -> None:
    """Write scalars on one line, each followed by a tab (core/io.py:94-120)."""
    fmt = _fmt(precision)
    with open(path, "w", newline="\n") as fh:
        fh.write("".join(fmt(float(v)) + "\t" for v in values))


def output_density_data_dat(density_flat, a: int, path: str, xlen: int, ylen: int, zlen: int,
                            precision: int = 32) -> None:
    """Write component a of a flattened grid (core/io.py:122-160)."""
    fmt = _fmt(precision)
    n = xlen * ylen * zlen
    d = np.asarray(density_flat, dtype=np.float64).reshape(-1)[a * n:(a + 1) * n].reshape(xlen, ylen, zlen)
    with open(path, "w", newline="\n") as fh:
        for x in range(xlen):
            fh.write(_rows(d[x], fmt))
            fh.write("\n")


def output_data_bundle_core(output_dir: str, *, h_Field, h_grid, xlen: int, ylen: int, zlen: int,
                            number_coordinates: int, number_total_fields: int, precision: int, bundle_spec,
                            arrays: dict, lattice_points_name: str = "LatticePoints.dat",
                            lattice_vectors_name: str = "LatticeVectors.dat",
                            field_dump_name: str = "d_Field.dat") -> None:
    """Lattice metadata, the whole field and one file per (array, component, name) of
    bundle_spec (core/io.py:162-246)."""
    os.makedirs(output_dir, exist_ok=True)
    n = xlen * ylen * zlen
    g = np.asarray(h_grid, dtype=np.float64).reshape(-1)
    last = (xlen - 1) * ylen * zlen + (ylen - 1) * zlen + (zlen - 1)
    ext = [float(g[c * n + last]) if number_coordinates > c else 0.0 for c in range(3)]
    points = np.array([xlen, ylen, zlen], dtype=np.float64)
    vectors = np.array([ext[0], 0.0, 0.0, 0.0, ext[1], 0.0, 0.0, 0.0, ext[2]], dtype=np.float64)
    output_iteration_data_dat(points[:number_coordinates], os.path.join(output_dir, lattice_points_name),
                              precision=precision)
    output_iteration_data_dat(vectors[:number_coordinates * number_coordinates],
                              os.path.join(output_dir, lattice_vectors_name), precision=precision)
    output_field_dat(h_Field, os.path.join(output_dir, field_dump_name), xlen, ylen, zlen, number_total_fields,
                     precision=precision)
    for key, a, filename in bundle_spec:
        arr = arrays.get(key)
        if arr is None:
            continue
        output_density_data_dat(arr, a, os.path.join(output_dir, filename), xlen, ylen, zlen, precision=precision)


# Per-theory bundles (th/*/io.py): grid coordinates, field components and densities.
_GRID = [("grid", 0, "xGrid.dat"), ("grid", 1, "yGrid.dat"), ("grid", 2, "zGrid.dat")]
_PION = [("Field", 0, "SigmaField.dat"), ("Field", 1, "PionField1.dat"), ("Field", 2, "PionField2.dat"),
         ("Field", 3, "PionField3.dat")]
_DENS = [("BaryonDensity", 0, "BaryonDensity.dat"), ("EnergyDensity", 0, "EnergyDensity.dat")]
BUNDLES = {
    "nuclear": _GRID + _PION + _DENS,
    "berger": _GRID + _PION + _DENS,
    "lightly_bound": _GRID + _PION + _DENS,
    "omega": _GRID + _PION + [("Field", 4, "OmegaMeson.dat")] + _DENS,
    "coulomb": _GRID + _PION + [("Field", 4, "CoulombField.dat")] + _DENS,
    "rho": _GRID + _PION + [("Field", 4 + 3 * i + a, f"Rho_{i + 1}_{a + 1}.dat") for i in range(3) for a in range(3)]
    + _DENS,
}


def make_output_data_bundle(short: str):
    """output_data_bundle of a theory's io module (th/*/io.py:13-100)."""
    spec = BUNDLES[short]

    def output_data_bundle(output_dir: str, h_Field, h_EnergyDensity, h_BaryonDensity, h_grid, xlen: int, ylen: int,
                           zlen: int, number_coordinates: int = 3, number_total_fields: int = 4,
                           precision: int = 32) -> None:
        arrays = {"grid": h_grid, "Field": h_Field, "EnergyDensity": h_EnergyDensity,
                  "BaryonDensity": h_BaryonDensity}
        output_data_bundle_core(output_dir, h_Field=h_Field, h_grid=h_grid, xlen=xlen, ylen=ylen, zlen=zlen,
                                number_coordinates=number_coordinates, number_total_fields=number_total_fields,
                                precision=precision, bundle_spec=spec, arrays=arrays,
                                lattice_points_name="LatticePoints.dat", lattice_vectors_name="LatticeVectors.dat",
                                field_dump_name="Field.dat")
    return output_data_bundle
