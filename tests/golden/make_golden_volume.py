"""Golden RGBA volume of the reference viewer, produced by the reference's own
kernels under Numba's CUDA simulator:
`python tests/golden/make_golden_volume.py`, after make_golden.py.

The viewer module (th/nuclear_skyrme/render_gl.py) imports its window and GL
libraries at the top, so it is not imported.  Its three CUDA kernels, which
use none of them (reduce_max_kernel :59-106, reduce_min_kernel :108-155,
build_rgba_volume_kernel :157-222), are taken from the module's source text
with `ast` and compiled in the simulator.  The multi-pass extrema follow
_reduce_density_extrema (:447-500): block reductions of 256 until one block
remains.

Inputs: `field0` and the reference's baryon density `baryon_density0` of
nuclear.npz (sim.en after compute_baryon_density, the density the viewer
shows).  Output: volume.npz with the extrema and the (Z, Y, X, 4) float32
volume.
"""
import ast
import math
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from tests.golden.make_golden import REFERENCE_ROOT, load_reference  # noqa: E402

KERNELS = ("reduce_max_kernel", "reduce_min_kernel", "build_rgba_volume_kernel")


def viewer_kernels():
    path = os.path.join(REFERENCE_ROOT, "skyrmion_solver", "theories", "nuclear_skyrme", "render_gl.py")
    tree = ast.parse(open(path).read())
    keep = [n for n in tree.body if isinstance(n, ast.FunctionDef) and n.name in KERNELS]
    block = [n for n in tree.body if isinstance(n, ast.Assign)
             and any(getattr(t, "id", None) == "_REDUCE_BLOCK_SIZE" for t in n.targets)]
    assert len(keep) == len(KERNELS) and len(block) == 1
    from numba import cuda, float64
    ns = {"cuda": cuda, "float64": float64, "math": math, "np": np}
    exec(compile(ast.Module(body=block + keep, type_ignores=[]), path, "exec"), ns)
    return ns


def main():
    load_reference()  # sets NUMBA_ENABLE_CUDASIM and patches the simulator
    from numba import cuda
    ns = viewer_kernels()
    bs = ns["_REDUCE_BLOCK_SIZE"]
    d = dict(np.load(os.path.join(HERE, "nuclear.npz")))
    X, Y, Z = (int(v) for v in d["p_i"][:3])
    dens = np.ascontiguousarray(d["baryon_density0"].ravel())
    field = np.ascontiguousarray(d["field0"].ravel())

    def reduce(kernel, values):
        cur = cuda.to_device(values)
        n = values.size
        while True:
            blocks = max(1, (n + bs - 1) // bs)
            out = cuda.device_array(blocks, dtype=np.float64)
            kernel[blocks, bs](cur, out, n)
            if blocks == 1:
                return out
            cur, n = out, blocks

    dmax = reduce(ns["reduce_max_kernel"], dens)
    dmin = reduce(ns["reduce_min_kernel"], dens)
    vol = cuda.device_array((Z, Y, X, 4), dtype=np.float32)
    block3d = (8, 8, 4)
    grid3d = tuple((n + b - 1) // b for n, b in zip((X, Y, Z), block3d))
    ns["build_rgba_volume_kernel"][grid3d, block3d](vol, cuda.to_device(dens), cuda.to_device(field), dmin, dmax,
                                                    X, Y, Z)
    out = dict(p_i=d["p_i"], density=dens, dmin=dmin.copy_to_host()[0], dmax=dmax.copy_to_host()[0],
               volume=vol.copy_to_host())
    np.savez_compressed(os.path.join(HERE, "volume.npz"), **out)
    print("extrema", out["dmin"], out["dmax"], "volume", out["volume"].shape, flush=True)


if __name__ == "__main__":
    main()
