"""Autotuner for the engine's per-instance tiling and plane staging.

The marching stage kernels split a lattice into (x-chunk, 8-row y, 32-column z)
tiles; the x-chunk sets how many tiles one launch has (and so how evenly they
spread over the 148 SMs) against how many halo planes each block re-reads.  The
planes of a tile are staged either by TMA box copies or by per-thread cp.async
copies, and an FP32 omega tile can run as z-pairs (16 x 8 threads, two z-sites
each, packed FP32x2 arithmetic) instead of one site per thread (32 x 8).
``sky_engine_add`` picks the chunk with a cost model and the staging from the
library options; this module measures instead: for one (theory, precision,
lattice shape, device) it admits a probe instance, times a few steps per
candidate (staging, chunk) with CUDA events on the engine's stream
(``Engine.time_stages``) and keeps the fastest.  Results are cached in a JSON
file so that a serving process tunes each shape once.

Tiling changes only the order of the per-tile energy partial sums, so a tuned
instance follows the same trajectory as an untuned one (``tests/test_march.py``);
the two stagings are bitwise identical and z-pairs agree to FP32 rounding
(``tests/test_tma.py``).
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


def candidate_stagings(engine, iid, theory, precision: str) -> list:
    """(tma, pair) stagings worth timing for an admitted instance: the admission's own, and
    when it stages by TMA also cp.async and (FP32 omega) z-pair tiles."""
    cur = engine.staging(iid)
    out = [cur]
    if cur[0]:
        for st in ((True, False), (True, True), (False, False)):
            if st in out or (st[1] and not (theory == "omega" and precision != "fp64")):
                continue
            out.append(st)
    return out


def tune(theory, p_i, p_f, precision: str = "fp32c", field=None, device: int = 0, cache: TuneCache | None = None,
         steps: int = 12) -> dict:
    """Best (staging, x-chunk) for one lattice shape; cached.  Returns {"xc", "tma", "pair",
    "ms_per_step", "timings"} (timings keyed "tma,pair,xc")."""
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
    packed = (np.asarray(p_i, np.int32), np.asarray(p_f, np.float64))
    with Engine(device) as eng:
        probe = eng.add(theory, packed, field, None, precision=precision)
        stagings = candidate_stagings(eng, probe, theory, precision)
        eng.remove(probe)
        t = {}
        # every candidate starts from the same field: a flow that has begun to arrest runs
        # cheaper steps (stage 2 skips an arrested step), which would favour later candidates
        for st in stagings:
            for xc in candidate_chunks(X):
                iid = eng.add(theory, packed, field, None, precision=precision)
                eng.set_staging(iid, *st)
                (got, ms), = time_chunks(eng, iid, [xc], steps=steps).items()
                t[(int(st[0]), int(st[1]), int(got))] = ms
                eng.remove(iid)
        best = min(t, key=t.get)
        res = {"xc": best[2], "tma": best[0], "pair": best[1], "ms_per_step": float(t[best]),
               "timings": {"%d,%d,%d" % k: v for k, v in t.items()}}
    cache.put(key, res)
    return res


def apply(engine, iid, theory, precision: str, p_i, cache: TuneCache | None = None, device: int = 0) -> bool:
    """Re-tile (and re-stage) `iid` with a cached choice for its shape, if one exists; returns
    whether it did.  A cached staging the instance cannot use (TMA switched off by option 2, or
    a lattice that breaks its alignment rule) is skipped; the chunk is still applied."""
    cache = cache if cache is not None else TuneCache()
    hit = cache.get(shape_key(theory, precision, p_i, _device_name(device)))
    if not hit or not hit.get("xc"):
        return False
    if "tma" in hit and (engine.staging(iid)[0] or not hit["tma"]):
        engine.set_staging(iid, bool(hit["tma"]), bool(hit.get("pair", 0)))
    engine.retile(iid, int(hit["xc"]))
    return True
