"""Autotuner for the engine's per-instance tiling.

The marching stage kernels split a lattice into (x-chunk, 8-row y, 32-column z)
tiles; the x-chunk sets how many tiles one launch has (and so how evenly they
spread over the 148 SMs) against how many halo planes each block re-reads.
``sky_engine_add`` picks it with a cost model; this module measures instead:
for one (theory, precision, lattice shape, device) it admits a probe instance,
times a few steps per candidate chunk with CUDA events on the engine's stream
(``Engine.time_stages``) and keeps the fastest.  Results are cached in a JSON
file so that a serving process tunes each shape once.

Tiling changes only the order of the per-tile energy partial sums, so a tuned
instance follows the same trajectory as an untuned one (``tests/test_march.py``).
"""
from __future__ import annotations

import json
import os
import threading

import numpy as np

DEFAULT_CACHE = os.environ.get("SKY_TUNE_CACHE", os.path.join(os.path.expanduser("~"), ".cache", "skyrmion_b200",
                                                              "tune.json"))


def candidate_chunks(X: int) -> list[int]:
    """x-chunks worth timing for a lattice of X planes (0 = the cost-model choice)."""
    c = {0, X}
    for k in (8, 12, 16, 20, 24, 32, 48, 64):
        if 4 <= k < X:
            c.add(k)
    for parts in (2, 3, 4, 6, 8):
        k = -(-X // parts)
        if 4 <= k < X:
            c.add(k)
    return sorted(c)


def shape_key(theory, precision: str, p_i, device_name: str) -> str:
    X, Y, Z = (int(v) for v in p_i[:3])
    return f"{device_name}|{theory}|{precision}|{X}x{Y}x{Z}"


class TuneCache:
    def __init__(self, path: str | None = DEFAULT_CACHE):
        self.path = path
        self.lock = threading.Lock()
        self.data = {}
        if path and os.path.exists(path):
            try:
                with open(path) as fh:
                    self.data = json.load(fh)
            except (OSError, ValueError):
                self.data = {}

    def get(self, key):
        return self.data.get(key)

    def put(self, key, value):
        with self.lock:
            self.data[key] = value
            if self.path:
                os.makedirs(os.path.dirname(self.path) or ".", exist_ok=True)
                tmp = self.path + ".tmp"
                with open(tmp, "w") as fh:
                    json.dump(self.data, fh, indent=1, sort_keys=True)
                os.replace(tmp, self.path)


def _device_name(device: int) -> str:
    import torch
    return torch.cuda.get_device_name(device).replace("|", "/")


def time_chunks(engine, iid, chunks, steps: int = 12, warm: int = 2) -> dict:
    """ms per step of instance `iid` (alone in `engine`) for each x-chunk."""
    out = {}
    for xc in chunks:
        engine.retile(iid, xc)
        engine.time_stages(warm)
        st = engine.time_stages(steps)
        out[engine.xc(iid)] = sum(st.values())
    return out


def tune(theory, p_i, p_f, precision: str = "fp32c", field=None, device: int = 0, cache: TuneCache | None = None,
         steps: int = 12) -> dict:
    """Best x-chunk for one lattice shape; cached.  Returns {"xc", "ms_per_step", "timings"}."""
    from .engine import Engine
    cache = cache if cache is not None else TuneCache()
    key = shape_key(theory, precision, p_i, _device_name(device))
    hit = cache.get(key)
    if hit is not None:
        return hit
    C, X, Y, Z = int(p_i[5]), int(p_i[0]), int(p_i[1]), int(p_i[2])
    if field is None:
        from .initial import exp_profile, hedgehog, with_extra_components
        h = (float(p_f[3]), float(p_f[4]), float(p_f[5]))
        field = with_extra_components(hedgehog((X, Y, Z), h, exp_profile(1.5)), C)
    with Engine(device) as eng:
        iid = eng.add(theory, (np.asarray(p_i, np.int32), np.asarray(p_f, np.float64)), field, None,
                      precision=precision)
        t = time_chunks(eng, iid, candidate_chunks(X), steps=steps)
        best = min(t, key=t.get)
        res = {"xc": int(best), "ms_per_step": float(t[best]), "timings": {str(k): v for k, v in t.items()}}
    cache.put(key, res)
    return res


def apply(engine, iid, theory, precision: str, p_i, cache: TuneCache | None = None, device: int = 0) -> bool:
    """Re-tile `iid` with a cached choice for its shape, if one exists; returns whether it did."""
    cache = cache if cache is not None else TuneCache()
    hit = cache.get(shape_key(theory, precision, p_i, _device_name(device)))
    if hit and hit.get("xc"):
        engine.retile(iid, int(hit["xc"]))
        return True
    return False
