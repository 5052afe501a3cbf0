"""Continuous-batching request loop over the resident engine.

Requests (one relaxation each: a theory, its packed parameters and an initial
FP64 field, or an initial configuration that is built on the device at
admission) arrive open-loop.  The loop:

* admits pending requests whose arrival time has passed, in arrival order,
  while the engine's device memory plus the request's estimate stays under the
  memory cap and the device keeps ``reserve_bytes`` free;
* advances every admitted instance together, ``chunk`` arrested-Newton steps at
  a time (graph-replayed launches, all theories and sizes in the same step);
* after each chunk reads every instance's latest statistics in one call and
  - switches an FP32 instance to FP64 once its gradient max-norm reaches
    ``switch_tol`` (by default ``switch_factor`` = 2 times the estimated FP32
    stencil noise floor, ``fp32_gradient_floor``) or has not improved by 1 % over
    ``plateau_chunks`` chunks, so the last digits are polished in FP64,
  - retires an instance whose FP64 gradient max-norm is at or below ``tol``
    (converged), whose energy is not finite (failed) or that used up
    ``max_steps`` (not converged), reading its field back and freeing its
    memory so that waiting requests can be admitted.

Time-to-converged is measured from a request's arrival to its retirement.
A request's trajectory does not depend on what else is in the batch (each
instance's reductions have a fixed order and the chunk boundaries are global),
so a result is the same alone and in the mix.
"""
from __future__ import annotations

import math
import time
from dataclasses import dataclass

import numpy as np


@dataclass
class Request:
    rid: int
    theory: str
    p_i: np.ndarray
    p_f: np.ndarray
    field: np.ndarray | None        # (C, X, Y, Z) FP64, reference layout; None: built from `init`
    arrival: float = 0.0            # seconds after the loop starts
    tol: float = 1e-6               # FP64 gradient max-norm at which the solve is converged
    max_steps: int = 1_000_000
    init: dict | None = None        # initial configuration built on the device at admission


@dataclass
class Result:
    rid: int
    status: str                     # "converged", "not_converged" or "failed"
    energy: float
    baryon: float
    gabs: float
    steps: int
    fp32_steps: int
    arrival: float
    admitted: float
    finished: float
    field: np.ndarray | None = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


def instance_bytes(C: int, N: int, precision: str = "fp32") -> int:
    """Device bytes of one engine instance: 7 state / slope arrays plus per-tile partials and the stats ring."""
    es = 4 if precision == "fp32" else 8
    return 7 * es * C * N + 8192 * 48 + (N // 256 + 1) * 48


def fp32_gradient_floor(p_f) -> float:
    """Estimated FP32 noise floor of the gradient max-norm on a lattice with spacings p_f[3:6].

    The second-difference stencil sums |coefficients| = 16/3 per axis over h^2, and a
    unit-size field is stored to 2^-24 relative, so an FP32 gradient carries errors
    of about 2^-24 * sum_i 16 / (3 h_i^2) (4.2e-5 at h = 0.15).
    """
    return 2.0 ** -24 * sum(16.0 / (3.0 * float(p_f[k]) ** 2) for k in (3, 4, 5))


class PlateauRule:
    """When to leave the FP32 phase: max|g| at or below `switch_tol` (by default twice the
    estimated FP32 noise floor), or no improvement by the factor `gain` over `window` steps."""

    def __init__(self, switch_tol: float = 0.0, window: int = 16384, gain: float = 0.99):
        self.switch_tol = switch_tol
        self.window = window
        self.gain = gain
        self.best = math.inf
        self.since = 0

    def update(self, gabs: float, steps: int) -> bool:
        if gabs < self.gain * self.best:
            self.best = gabs
            self.since = 0
        else:
            self.since += steps
        return gabs <= self.switch_tol or self.since >= self.window


@dataclass
class _Live:
    req: Request
    iid: int
    precision: str
    admitted: float
    fp32_steps: int = 0
    rule: PlateauRule | None = None


class Server:
    """Continuous batching of relaxation requests on one GPU.

    ``engine`` is a ``skyrmion_solver_b200.engine.Engine`` (or an object with the
    same methods); ``free_bytes`` returns the device's free memory (defaults to
    ``torch.cuda.mem_get_info``); ``clock`` returns seconds.
    """

    def __init__(self, engine, mem_cap_bytes: float = 180e9, reserve_bytes: float = 2e9, chunk: int = 64,
                 switch_tol: float | None = None, plateau_chunks: int = 256, plateau_gain: float = 0.99,
                 polish: bool = True,
                 keep_fields: bool = True, free_bytes=None, clock=time.perf_counter, sleep=time.sleep,
                 fp32_mode: str = "fp32d", tune_cache=None, defect_period: int | None = None,
                 switch_factor: float = 2.0):
        self.engine = engine
        self.mem_cap = float(mem_cap_bytes)
        self.reserve = float(reserve_bytes)
        self.chunk = int(chunk)
        self.switch_tol = switch_tol   # None: switch_factor x the request's estimated FP32 gradient floor
        self.switch_factor = float(switch_factor)
        self.plateau_chunks = int(plateau_chunks)
        self.plateau_gain = float(plateau_gain)
        self.polish = polish
        # "fp32d" (compensated, defect-corrected), "fp32c" (compensated), "fp32", or "fp64" (no FP32 phase)
        self.fp32_mode = fp32_mode
        # autotune.TuneCache: re-stage and re-tile admitted instances with cached per-shape choices
        # (tuned for an instance alone; in a full batch the admission's chunks measured faster)
        self.tune_cache = tune_cache
        self.keep_fields = keep_fields
        self.defect_period = defect_period  # refresh period of fp32d corrections (None: the engine's 16)
        self.clock = clock
        self.sleep = sleep
        if free_bytes is None:
            def free_bytes():
                import torch
                return torch.cuda.mem_get_info(engine.device)[0]
        self.free_bytes = free_bytes
        self.pending: list[Request] = []
        self.live: dict[int, _Live] = {}
        self.results: list[Result] = []
        self.t0 = None
        self.steps_run = 0

    # ------------------------------------------------------------------
    def submit(self, req: Request):
        self.pending.append(req)
        self.pending.sort(key=lambda r: (r.arrival, r.rid))

    def now(self) -> float:
        return self.clock() - self.t0

    def _admit(self):
        t = self.now()
        while self.pending and self.pending[0].arrival <= t:
            req = self.pending[0]
            C, N = int(req.p_i[5]), int(req.p_i[6])
            need = instance_bytes(C, N, "fp64" if self.polish else "fp32")
            if self.live and (self.engine.bytes + need > self.mem_cap or self.free_bytes() - need < self.reserve):
                break                                   # wait for a retirement to free memory
            self.pending.pop(0)
            try:
                field = req.field if req.field is not None else self._device_field(req)
                iid = self.engine.add(req.theory, (req.p_i, req.p_f), field, None, precision=self.fp32_mode)
            except MemoryError:
                self.results.append(Result(req.rid, "failed", math.nan, math.nan, math.nan, 0, 0, req.arrival, t,
                                           t))
                continue
            if self.defect_period is not None and self.fp32_mode == "fp32d":
                self.engine.set_defect_period(iid, self.defect_period)
            if self.tune_cache is not None:
                from .autotune import apply
                apply(self.engine, iid, req.theory, self.fp32_mode, req.p_i, self.tune_cache, self.engine.device)
            self.live[iid] = _Live(req, iid, "fp64" if self.fp32_mode == "fp64" else "fp32", t,
                                   rule=PlateauRule(self._switch_tol(req), self.plateau_chunks * self.chunk,
                                                    self.plateau_gain))

    def _device_field(self, req: Request):
        """The request's initial field built on the engine's device (sky_init_field), with the
        omega component seeded as -c_omega B0 for the omega variant; no host field is made."""
        from .theories._init_common import build_device_field, seed_omega
        f = build_device_field(req.theory, req.p_i, req.p_f, req.init or {}, device=self.engine.device)
        if req.theory == "omega" and (req.init or {}).get("omega_seed", True):
            seed_omega(f, req.p_i, req.p_f)
        return f

    def _switch_tol(self, req: Request) -> float:
        if self.switch_tol is not None:
            return float(self.switch_tol)
        if self.fp32_mode == "fp32d":      # the corrected gradient reaches the tolerance itself
            return req.tol
        return self.switch_factor * fp32_gradient_floor(req.p_f)

    def _retire(self, lv: _Live, st, status: str):
        f = None
        if self.keep_fields:
            f, _ = self.engine.read(lv.iid, velocity=False)
        self.engine.remove(lv.iid)
        del self.live[lv.iid]
        self.results.append(Result(lv.req.rid, status, st.energy, st.baryon, st.gabs, st.step,
                                   lv.fp32_steps if lv.precision == "fp64" else st.step, lv.req.arrival,
                                   lv.admitted, self.now(), f))

    def _review(self):
        stats = self.engine.stats_all()
        for iid, lv in list(self.live.items()):
            st = stats[iid]
            if not (math.isfinite(st.energy) and math.isfinite(st.gabs)):
                self._retire(lv, st, "failed")
                continue
            if lv.precision == "fp64" or not self.polish:
                if st.gabs <= lv.req.tol:
                    self._retire(lv, st, "converged")
                    continue
            else:
                # FP32 phase: switch to FP64 at switch_tol or when max|g| stops improving
                if lv.rule.update(st.gabs, self.chunk) or st.gabs <= lv.req.tol:
                    self.engine.set_precision(iid, "fp64")
                    lv.precision = "fp64"
                    lv.fp32_steps = st.step
            if st.step >= lv.req.max_steps:
                self._retire(lv, st, "not_converged")

    def run(self, until_idle: bool = True, time_limit: float | None = None):
        """Serve until every submitted request is retired (or time_limit seconds pass)."""
        if self.t0 is None:
            self.t0 = self.clock()
        while self.pending or self.live:
            if time_limit is not None and self.now() > time_limit:
                break
            self._admit()
            if not self.live:
                if not self.pending:
                    break
                wait = self.pending[0].arrival - self.now()     # idle until the next arrival
                if wait > 0:
                    self.sleep(min(wait, 0.01))
                continue
            self.engine.step(self.chunk)
            self.steps_run += self.chunk
            self._review()
        return self.results

    # ------------------------------------------------------------------
    def summary(self) -> dict:
        lat = np.array([r.latency for r in self.results if r.status == "converged"])
        span = max((r.finished for r in self.results), default=0.0)
        done = int(lat.size)
        return {
            "requests": len(self.results),
            "converged": done,
            "failed": sum(r.status == "failed" for r in self.results),
            "not_converged": sum(r.status == "not_converged" for r in self.results),
            "solves_per_s": done / span if span > 0 else None,
            "p50_s": float(np.percentile(lat, 50)) if done else None,
            "p99_s": float(np.percentile(lat, 99)) if done else None,
            "wall_s": span,
            "batch_steps": self.steps_run,
        }


def poisson_arrivals(rate: float, n: int, seed: int = 0) -> np.ndarray:
    """Open-loop Poisson arrival times (seconds) of n requests at `rate` per second."""
    rng = np.random.default_rng(seed)
    return np.cumsum(rng.exponential(1.0 / rate, size=n))
