"""Continuous-batching request loop (skyrmion_solver_b200.serving).

CPU tests drive the loop with a fake engine and a fake clock: arrival order,
admission under the memory cap, the FP32 -> FP64 switch on a gradient plateau,
retirement (converged / failed / step limit) and the latency summary.  The GPU
test checks on the B200 that a request's result is the same served alone and
served in a mix of other theories and sizes (bitwise: each instance's
trajectory is independent of the batch).
"""
import math
from dataclasses import dataclass

import numpy as np
import pytest

from skyrmion_solver_b200.serving import Request, Server, instance_bytes, poisson_arrivals


@dataclass
class _St:
    energy: float
    baryon: float
    err: float
    gabs: float
    arrested: bool
    step: int
    precision: str


class FakeEngine:
    """Each instance's max|g| decays by `rate` per step down to a precision floor (1e-5 in FP32)."""

    def __init__(self, clock, step_cost=1e-4, rate=0.99, fp32_floor=1e-5):
        self.clock = clock
        self.step_cost = step_cost
        self.rate = rate
        self.fp32_floor = fp32_floor
        self.insts = {}
        self.next = 0
        self.device = 0
        self.max_bytes = 0
        self.switches = []

    @property
    def bytes(self):
        return sum(v["bytes"] for v in self.insts.values())

    def add(self, theory, params, field, velocity=None, precision="fp32"):
        p_i = params[0]
        C, N = int(p_i[5]), int(p_i[6])
        iid = self.next
        self.next += 1
        self.insts[iid] = dict(g=1.0, step=0, prec=precision, bytes=instance_bytes(C, N, "fp64"),
                               nan=theory == "nan", field=np.asarray(field))
        self.max_bytes = max(self.max_bytes, self.bytes)
        return iid

    def step(self, n):
        self.clock.t += n * self.step_cost * max(1, len(self.insts))
        for v in self.insts.values():
            v["step"] += n
            floor = self.fp32_floor if v["prec"] != "fp64" else 0.0
            v["g"] = max(floor, v["g"] * self.rate ** n)

    def stats_all(self):
        out = {}
        for i, v in self.insts.items():
            e = math.nan if v["nan"] and v["step"] > 100 else 1.0 + v["g"]
            out[i] = _St(e, 1.0, v["g"], v["g"], False, v["step"], v["prec"])
        return out

    def set_precision(self, iid, precision):
        self.insts[iid]["prec"] = precision
        self.switches.append((iid, self.insts[iid]["step"]))

    def read(self, iid, velocity=True):
        return self.insts[iid]["field"], None

    def remove(self, iid):
        del self.insts[iid]


class FakeClock:
    def __init__(self):
        self.t = 0.0

    def __call__(self):
        return self.t

    def sleep(self, dt):
        self.t += dt


def _req(rid, arrival, C=4, L=16, theory="nuclear", tol=1e-6, max_steps=10 ** 6):
    p_i = np.array([L, L, L, 2, 3, C, L ** 3, C * L ** 3, 1, 1, 1], np.int32)
    p_f = np.array([0.0, 0.0, 0.0, 0.2, 0.2, 0.2, 0.008, 0.02])
    return Request(rid, theory, p_i, p_f, np.zeros((C, L, L, L)), arrival, tol, max_steps)


def test_all_requests_converge_with_fp64_polish():
    clk = FakeClock()
    eng = FakeEngine(clk)
    srv = Server(eng, mem_cap_bytes=1e12, reserve_bytes=0, chunk=16, plateau_chunks=4, free_bytes=lambda: 1e12,
                 clock=clk, sleep=clk.sleep)
    for k, t in enumerate(poisson_arrivals(50.0, 12, seed=1)):
        srv.submit(_req(k, float(t)))
    res = srv.run()
    assert len(res) == 12 and all(r.status == "converged" for r in res)
    assert all(r.gabs <= 1e-6 for r in res)
    # every instance switched to FP64 once its FP32 gradient stalled at the floor
    assert len(eng.switches) == 12
    assert all(0 < r.fp32_steps < r.steps for r in res)
    assert all(r.admitted >= r.arrival for r in res)
    s = srv.summary()
    assert s["converged"] == 12 and s["p50_s"] <= s["p99_s"] and s["solves_per_s"] > 0


def test_admission_respects_memory_cap():
    clk = FakeClock()
    eng = FakeEngine(clk)
    one = instance_bytes(4, 16 ** 3, "fp64")
    srv = Server(eng, mem_cap_bytes=2.5 * one, reserve_bytes=0, chunk=32, plateau_chunks=2,
                 free_bytes=lambda: 1e12, clock=clk, sleep=clk.sleep)
    for k in range(7):
        srv.submit(_req(k, 0.0))
    res = srv.run()
    assert len(res) == 7 and all(r.status == "converged" for r in res)
    assert eng.max_bytes <= 2.5 * one
    # requests are admitted in arrival order and later ones wait for retirements
    adm = sorted(res, key=lambda r: r.rid)
    assert adm[0].admitted <= adm[-1].admitted and adm[-1].admitted > 0.0


def test_arrival_order_and_open_loop_idle():
    clk = FakeClock()
    eng = FakeEngine(clk)
    srv = Server(eng, mem_cap_bytes=1e12, reserve_bytes=0, chunk=16, plateau_chunks=2, free_bytes=lambda: 1e12,
                 clock=clk, sleep=clk.sleep)
    srv.submit(_req(0, 5.0))   # arrives after an idle gap
    srv.submit(_req(1, 0.0))
    res = {r.rid: r for r in srv.run()}
    assert res[0].admitted >= 5.0
    assert res[1].admitted < 5.0


def test_failures_and_step_limit():
    clk = FakeClock()
    eng = FakeEngine(clk, rate=0.999999)
    srv = Server(eng, mem_cap_bytes=1e12, reserve_bytes=0, chunk=64, free_bytes=lambda: 1e12, clock=clk,
                 sleep=clk.sleep)
    srv.submit(_req(0, 0.0, theory="nan"))
    srv.submit(_req(1, 0.0, max_steps=640))
    res = {r.rid: r for r in srv.run()}
    assert res[0].status == "failed"
    assert res[1].status == "not_converged" and res[1].steps >= 640
    assert srv.summary()["converged"] == 0


def test_fp32_floor_estimate():
    from skyrmion_solver_b200.serving import fp32_gradient_floor
    f = fp32_gradient_floor([0, 0, 0, 0.15, 0.15, 0.15])
    assert 4.0e-5 < f < 4.5e-5          # the plateau observed for FP32 omega solves at h = 0.15


def test_poisson_arrivals_rate():
    t = poisson_arrivals(20.0, 4000, seed=3)
    assert np.all(np.diff(t) > 0)
    assert abs(len(t) / t[-1] - 20.0) < 1.5


# ---------------------------------------------------------------------------
# GPU: alone vs in the mix
# ---------------------------------------------------------------------------

def _gpu_request(rid, name, dims, seed, tol=2e-4):
    from tests.test_march import inputs, params_for
    th, p_i, p_f = params_for(name, dims)
    F, _ = inputs(int(p_i[5]), dims, seed=seed)
    return Request(rid, name, p_i, p_f, F, 0.0, tol, 6000)


@pytest.mark.gpu
def test_result_same_alone_and_in_mix():
    from skyrmion_solver_b200.engine import Engine
    target = dict(name="nuclear", dims=(24, 20, 28), seed=11)
    with Engine(0) as eng:
        srv = Server(eng, chunk=32, plateau_chunks=4)
        srv.submit(_gpu_request(0, **target))
        alone = srv.run()[0]
    with Engine(0) as eng:
        srv = Server(eng, chunk=32, plateau_chunks=4)
        srv.submit(_gpu_request(0, **target))
        srv.submit(_gpu_request(1, "omega", (20, 26, 18), 12))
        srv.submit(_gpu_request(2, "coulomb", (22, 18, 24), 13))
        srv.submit(_gpu_request(3, "nuclear", (30, 16, 20), 14))
        mix = {r.rid: r for r in srv.run()}[0]
    assert alone.status == mix.status
    assert (alone.steps, alone.fp32_steps) == (mix.steps, mix.fp32_steps)
    assert alone.energy == mix.energy and alone.gabs == mix.gabs
    assert np.array_equal(alone.field, mix.field)


def test_tune_cache_roundtrip(tmp_path):
    from skyrmion_solver_b200.autotune import TuneCache, candidate_chunks, shape_key
    path = str(tmp_path / "tune.json")
    c = TuneCache(path)
    p_i = np.array([128, 128, 128, 2, 3, 5, 128 ** 3, 5 * 128 ** 3, 1, 1, 1, 4], np.int32)
    k = shape_key("omega", "fp32c", p_i, "NVIDIA B200")
    assert c.get(k) is None
    c.put(k, {"xc": 32, "ms_per_step": 0.5, "timings": {"32": 0.5}})
    assert TuneCache(path).get(k)["xc"] == 32
    ch = candidate_chunks(128)
    assert 0 in ch and 128 in ch and 32 in ch and all(0 <= x <= 128 for x in ch)
    assert candidate_chunks(5) == [0, 5]


@pytest.mark.gpu
def test_autotune_picks_a_measured_chunk(tmp_path):
    from skyrmion_solver_b200 import autotune
    from tests.test_march import params_for
    th, p_i, p_f = params_for("omega", (40, 24, 36))
    cache = autotune.TuneCache(str(tmp_path / "tune.json"))
    res = autotune.tune("omega", p_i, p_f, "fp32c", cache=cache, steps=4)
    keys = [tuple(int(v) for v in k.split(",")) for k in res["timings"]]
    assert (res["tma"], res["pair"], res["xc"]) in keys
    assert {(k[0], k[1]) for k in keys} == {(1, 0), (1, 1), (0, 0)}   # TMA, z-pairs, cp.async
    assert res["ms_per_step"] == min(res["timings"].values())
    assert autotune.tune("omega", p_i, p_f, "fp32c", cache=cache) == res      # cached
    from skyrmion_solver_b200.engine import Engine
    from tests.test_march import inputs
    F, _ = inputs(int(p_i[5]), (40, 24, 36), seed=3)
    with Engine(0) as eng:
        i = eng.add("omega", (p_i, p_f), F, None, precision="fp32c")
        assert autotune.apply(eng, i, "omega", "fp32c", p_i, cache)
        assert eng.staging(i) == (bool(res["tma"]), bool(res["pair"])) and eng.xc(i) == res["xc"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["nuclear", "omega"])
def test_request_built_on_the_device(name):
    """A request that carries an initial configuration instead of a field is built on the
    device at admission (omega seeded there too): the solve is bitwise the one of a request
    that carries that same field from the host.  (The device builder itself is checked
    against the host builder in tests/test_init.py; tiny input differences are not compared
    through a solve, since the arrest decisions of the omega flow amplify them.)"""
    import torch
    from skyrmion_solver_b200.engine import Engine
    from skyrmion_solver_b200.theories._init_common import build_device_field, seed_omega
    from tests.test_march import params_for
    th, p_i, p_f = params_for(name, (24, 22, 26))
    cfg = {"mode": "hedgehog", "scale": 1.0, "center": (0.1, -0.1, 0.05), "vacuum_shell": 2}
    t = build_device_field(name, p_i, p_f, cfg)
    if name == "omega":
        seed_omega(t, p_i, p_f)
    torch.cuda.synchronize()
    host = t.cpu().numpy().reshape((int(p_i[5]),) + tuple(int(v) for v in p_i[:3]))
    out = {}
    for key, req in (("host", Request(0, name, p_i, p_f, host, 0.0, 2e-4, 2000)),
                     ("device", Request(0, name, p_i, p_f, None, 0.0, 2e-4, 2000, init=cfg))):
        with Engine(0) as eng:
            srv = Server(eng, chunk=32, plateau_chunks=4)
            srv.submit(req)
            out[key] = srv.run()[0]
    a, b = out["host"], out["device"]
    assert (a.status, a.steps, a.fp32_steps) == (b.status, b.steps, b.fp32_steps)
    assert a.energy == b.energy and a.gabs == b.gabs
    assert np.array_equal(a.field, b.field)
