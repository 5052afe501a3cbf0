#!/usr/bin/env python
"""Benchmark of the lattice engine on the omega-meson B=4 relaxation (128^3, h = 0.15).

Workload: the pion + omega-meson Skyrme variant (5 components), B = 4 cubic
rational-map initial field with profile f(r) = pi exp(-r/2), 128^3 sites,
spacing 0.15, time step 0.2 h, two-site vacuum shell, omega seeded as
-c_omega B0, couplings of the reference's omega example (f_pi = 139.8,
m_pi = 43.91, m_omega = 249.5, beta_omega = 8.036: mass 0.176, c_omega 14.34).
State and stage arithmetic are FP32; energies, baryon numbers and the arrest
test are FP64 with compensated summation.

One bench step is one arrested-Newton step (four fused gradient stages, the RK4
update with projection onto S^3, FP64 energy / baryon reductions and the
device-side arrest decision) of the resident engine, replayed from CUDA graphs.

The headline unit is converged solves/s of the schedule the engine serves with:
compensated FP32 steps until the gradient max-norm stops improving, then FP64
steps, until the energy stays within 1e-6 relative of the converged plain-FP64
energy (the FP64 solve run to gradient max-norm <= 1e-6).  A solve takes
S32 * t32 + S64 * t64, with the step times t32 (the timed K steps) and t64
(the FP64 engine) measured in this run and the step counts S32, S64 measured on
the GPU by ``python bench.py --calibrate`` (``profiles/convergence_omega_B4_128.json``);
without that file the value is null.

Usage::

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python bench.py --calibrate          # full FP64 and FP32 solves, writes the step counts
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "converged solves/s and p99 latency at 1e-6 rel. energy vs plain FP64; HBM GB/s"
UNIT = "solves/s"
WORKLOAD = "omega_B4_rational_map_128^3_h0.15"
CALIBRATION = os.path.join(ROOT, "profiles", "convergence_omega_B4_128.json")
TRAFFIC = [os.path.join(ROOT, "profiles", f) for f in ("ncu_stage1_fp32d_omega128.md",
                                                        "ncu_stage4_fp32d_omega128.md")]
L = 128
H = 0.15
FAST = "fp32d"   # precision of the timed steps (the FP32 phase of the schedule)
SCHEDULE = {"fp32c": "mixed", "fp32d": "defect"}[FAST]   # its calibration entry
DT_FACTOR = 0.2
COUPLINGS = dict(f_pi=139.8, m_pi=43.91, m_omega=249.5, beta_omega=8.036)
INIT = {"mode": "rational_map", "baryon_number": 4, "scale": 2.0, "vacuum_shell": 2}
REL_ENERGY_TOL = 1e-6
GRAD_TOL = 1e-6
# passes over one C-component field per stage launch (reads + writes)
STAGE_PASSES = {"stage1": 2, "stage2": 3, "stage3": 4, "stage4": 7}


def stage_passes(stage, precision):
    """Field-sized passes (reads + writes of one C-component FP32 array) of one stage launch.
    Compensated field (fp32c, fp32d): stage 1 also reads the low parts (FP64 densities of hi + lo),
    stage 4 reads and writes them.  fp32d: every stage reads the correction; every 16th step the
    defect kernel reads hi and lo and writes it, and stage 1 rewrites it (4/16 per step, counted
    with stage 1, whose timing includes the defect kernel)."""
    n = STAGE_PASSES[stage]
    if precision in ("fp32c", "fp32d"):
        n += {"stage1": 1, "stage4": 2}.get(stage, 0)
    if precision == "fp32d":
        n += 1 + (4 / 16 if stage == "stage1" else 0)
    return n


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------

def workload_params():
    import numpy as np
    from skyrmion_solver_b200 import theories as T
    th = T.by_short_name("omega")
    p = th.params.default_params(xlen=L, ylen=L, zlen=L, lsx=H, lsy=H, lsz=H, xsize=H * (L - 1),
                                 ysize=H * (L - 1), zsize=H * (L - 1), time_step=DT_FACTOR * H, **COUPLINGS)
    p_i, p_f = th.params.pack_device_params(p.resolved())
    return th, p, np.asarray(p_i, dtype=np.int32), np.asarray(p_f, dtype=np.float64)


def workload_field_device(p_i, p_f, device):
    """Initial field on the device (FP64, reference layout), omega seeded by the library's own kernel."""
    import torch
    from skyrmion_solver_b200.theories._init_common import build_host_field, seed_omega
    f = build_host_field("omega", p_i, p_f, INIT)
    t = torch.from_numpy(f.ravel()).to(device)
    seed_omega(t, p_i, p_f)
    return t


def load_calibration():
    if not os.path.exists(CALIBRATION):
        return None
    with open(CALIBRATION) as fh:
        return json.load(fh)


def load_issue_active(stage):
    """smsp__issue_active (fraction of cycles a scheduler issued) of one stage kernel from the
    committed ncu summary, or None: the compute-side roofline of an issue-bound kernel."""
    import re
    for path in TRAFFIC:
        if os.path.exists(path):
            m = re.search(r"issue_active\[%s\]:\s*([0-9.eE+]+)" % stage, open(path).read())
            if m:
                return float(m.group(1))
    return None


def load_traffic(stage):
    """Per-launch DRAM bytes (read + write) of one stage kernel from the committed ncu summary, or None."""
    import re
    for path in TRAFFIC:
        if os.path.exists(path):
            m = re.search(r"traffic_bytes_per_launch\[%s\]:\s*([0-9.eE+]+)" % stage, open(path).read())
            if m:
                return float(m.group(1))
    return None


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------

class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.proc = None
        self.path = None
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(gpu_index), "--query-gpu=timestamp," + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.fh, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        self.t_start = self.t_end = None

    def mark_start(self):
        self.t_start = time.time()

    def mark_end(self):
        self.t_end = time.time()

    def stop(self):
        if self.proc is None:
            return {"unavailable": "nvidia-smi not found"}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.fh.close()
        rows = []
        for line in open(self.path):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                ts = time.mktime(time.strptime(parts[0].split(".")[0], "%Y/%m/%d %H:%M:%S"))
                rows.append((ts, float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        os.unlink(self.path)
        if not rows:
            return {"unavailable": "no samples"}
        lo = (self.t_start or 0) - 1.0
        hi = (self.t_end or 1e18) + 1.0
        win = [r for r in rows if lo <= r[0] <= hi] or rows
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[i] for r in win for i, v in enumerate(r[3]) if v.lower().startswith("active")})
        return {"sm_mhz": statistics.median(r[1] for r in win), "sm_max_mhz": max(r[2] for r in win),
                "reasons": reasons, "samples": len(win)}


# ---------------------------------------------------------------------------
# CPU baseline: the FP64 NumPy oracle on all host cores (one process per core)
# ---------------------------------------------------------------------------

def _cpu_worker(args):
    sub, nsteps, barrier, q = args
    os.environ["OMP_NUM_THREADS"] = "1"
    import numpy as np
    from oracle import skyrme_oracle as O
    th = O.THEORIES["omega"]
    F, V, p_i, p_f = sub
    E = O.total_energy(th, F, p_i, p_f)
    barrier.wait()
    t0 = time.perf_counter()
    for _ in range(nsteps):
        F, V, E, err, _ = O.arrested_newton_step(th, F, V, p_i, p_f, E)
    q.put((int(F[0].size) * nsteps, time.perf_counter() - t0))


def cpu_sample_inputs(side=64):
    """Central side^3 crop of the workload field, as its own lattice (same couplings, spacing, dt)."""
    import numpy as np
    from oracle import skyrme_oracle as O
    from skyrmion_solver_b200.theories._init_common import build_host_field
    th, p, p_i, p_f = workload_params()
    F = build_host_field("omega", p_i, p_f, INIT)
    N = int(p_i[6])
    b = O.baryon_density(O.THEORIES["omega"], F, p_i, p_f)
    F[4] = -float(p_f[9]) * b / float(p_f[6])
    o = (L - side) // 2
    Fc = np.ascontiguousarray(F[:, o:o + side, o:o + side, o:o + side])
    p_i2 = p_i.copy()
    p_i2[0:3] = side
    p_i2[6] = side ** 3
    p_i2[7] = int(p_i2[5]) * side ** 3
    return Fc, np.zeros_like(Fc), p_i2, p_f


def cpu_baseline(nsteps=2, side=64, max_procs=64):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    procs = max(1, min(os.cpu_count() or 1, max_procs))
    sub = cpu_sample_inputs(side)
    barrier = ctx.Barrier(procs)
    q = ctx.Queue()
    ps = [ctx.Process(target=_cpu_worker, args=((sub, nsteps, barrier, q),)) for _ in range(procs)]
    for pr in ps:
        pr.start()
    res = [q.get() for _ in ps]
    for pr in ps:
        pr.join()
    site_steps = sum(r[0] for r in res)
    secs = max(r[1] for r in res)
    return dict(site_steps_per_s=site_steps / secs, cores=procs, secs=secs,
                sample=f"{procs} processes x {nsteps} FP64 oracle arrested-Newton steps on a central {side}^3 crop "
                       f"of the workload field ({site_steps} site-steps in {secs:.1f} s)")


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------

def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def emit(obj):
    print(json.dumps(obj), flush=True)


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------

def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    cal = load_calibration()
    cb = cpu_baseline()
    N = L ** 3
    steps_per_s = cb["site_steps_per_s"] / N
    # the plain FP64 solve to max|g| <= 1e-6 takes 119,000 steps (FP64 engine on a B200; the CPU port runs
    # the same arithmetic, so the same step count), far more than a CPU run can time
    s64 = cal["fp64_total_steps"] if cal else None
    value = steps_per_s / s64 if s64 else None
    emit({"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
          "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
          "vs_baseline": None, "dtype": "f64", "data": "synthetic",
          "config": {"workload": WORKLOAD, "sites": N, "precision": "fp64 (oracle)",
                     "steps_to_converge": s64, "site_steps_per_s": cb["site_steps_per_s"]},
          "cpu_baseline": {"value": value, "unit": UNIT, "cores": cb["cores"], "kind": "port",
                           "sample": cb["sample"]},
          "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}})
    return 0


# ---------------------------------------------------------------------------
# the reference's own Numba-CUDA run on this GPU (installed under baseline/_ref)
# ---------------------------------------------------------------------------

NUMBA_STEPS = 3        # reference steps compared step by step with the drop-in path
NUMBA_TIMED = 10       # reference steps timed after them


def run_numba_reference(args):
    """Worker: the reference's unmodified Simulation (core/simulation.py:287-308, do_arrested_newton_flow of
    core/integrator.py:284-410) with its own omega theory kernels, compiled by Numba for this GPU, on the
    workload field read from args.field.  Prints one JSON line: per-step (energy, err) of the first
    NUMBA_STEPS steps, the wall time per step of NUMBA_TIMED more (each step ends in cuda.synchronize)."""
    import numpy as np
    out = {"impl": "reference-numba-cuda", "workload": WORKLOAD}
    try:
        from tests import _reference as R
        if not R.available():
            raise RuntimeError("the reference is not installed under baseline/_ref")
        from numba import cuda
        theories, Simulation, _ = R.load(("omega",))
        th = theories["omega"]
        p = th.params.Params(xlen=L, ylen=L, zlen=L, lsx=H, lsy=H, lsz=H, xsize=H * (L - 1), ysize=H * (L - 1),
                             zsize=H * (L - 1), time_step=DT_FACTOR * H, **COUPLINGS)
        sim = Simulation(p, th)
        field = np.load(args.field)
        sim.Field.copy_to_device(np.ascontiguousarray(field.ravel()))
        sim.Velocity.copy_to_device(np.zeros(field.size))
        e = sim.observables()["energy"]
        out["energy0"] = e
        t0 = time.perf_counter()
        steps = []
        for _ in range(NUMBA_STEPS):       # the first includes Numba's compilation of every kernel
            e, err = sim.step(e)
            steps.append((float(e), float(err)))
        cuda.synchronize()
        out["first_steps_s"] = time.perf_counter() - t0
        out["steps"] = steps
        t0 = time.perf_counter()
        for _ in range(NUMBA_TIMED):
            e, err = sim.step(e)
        cuda.synchronize()
        out["ms_per_step"] = (time.perf_counter() - t0) * 1e3 / NUMBA_TIMED
        out["timed_steps"] = NUMBA_TIMED
        out["device"] = cuda.get_current_device().name.decode() if isinstance(
            cuda.get_current_device().name, bytes) else str(cuda.get_current_device().name)
    except Exception as ex:  # reported as unavailable, with the reason
        out["unavailable"] = f"{type(ex).__name__}: {ex}"[:400]
    emit(out)
    return 0


def numba_reference_record(field, p, th, timeout_s=900):
    """Run the Numba-CUDA reference on `field` in a child process and compare its first steps with the
    drop-in path (this package's FP64 reference-layout kernels) from the same field."""
    import numpy as np
    import torch
    from skyrmion_solver_b200.core.simulation import Simulation
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "field.npy")
        np.save(path, field.detach().cpu().numpy())
        try:
            r = subprocess.run([sys.executable, os.path.abspath(__file__), "--numba-reference", "--field", path],
                               capture_output=True, text=True, timeout=timeout_s, cwd=ROOT)
            lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
            rec = json.loads(lines[-1]) if lines else {"unavailable": (r.stderr or r.stdout)[-400:]}
        except subprocess.TimeoutExpired:
            rec = {"unavailable": f"the reference's Numba-CUDA run did not finish within {timeout_s} s"}
    if "steps" in rec:
        sim = Simulation(p, th)
        sim.Field.copy_(field)
        sim.Velocity.zero_()
        e = sim.observables()["energy"]
        rel = [abs(e - rec["energy0"]) / abs(rec["energy0"])]
        for (er, errr) in rec["steps"]:
            e, err = sim.step(e)
            rel.append(abs(e - er) / abs(er))
        torch.cuda.synchronize()
        rec["drop_in_max_rel_energy_diff"] = max(rel)
        rec["drop_in_energy_diffs"] = rel
        del sim
    return rec


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------

def solve_to_tolerance(eng, iid, stream, chunk, max_steps, tol=GRAD_TOL):
    """Advance instance `iid` in chunks of `chunk` steps, reading its latest statistics (one
    64-byte device->host read) after each chunk, until max|g| <= tol; a defect-corrected or
    compensated FP32 instance whose gradient stops improving by 1 % over 16,384 steps switches to
    FP64 first (the serving rule).  Returns (stats, steps, fp32 steps, device ms, wall s)."""
    import torch
    from skyrmion_solver_b200.serving import PlateauRule
    rule = PlateauRule(tol)
    prec = eng.meta[iid]["precision"]
    fp32_steps = 0
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    ev0.record(stream)
    n = 0
    st = eng.stats(iid)
    while n < max_steps:
        eng.step(chunk)
        n += chunk
        st = eng.stats(iid)
        if not math.isfinite(st.energy):
            break
        if prec == "fp64" or eng.meta[iid]["precision"] == "fp64":
            if st.gabs <= tol:
                break
        elif st.gabs <= tol:
            break
        elif rule.update(st.gabs, chunk):
            eng.set_precision(iid, "fp64")
            fp32_steps = n
    ev1.record(stream)
    ev1.synchronize()
    wall = time.perf_counter() - t0
    if eng.meta[iid]["precision"] != "fp64":
        fp32_steps = n
    return st, n, fp32_steps, ev0.elapsed_time(ev1), wall


def run_ours(args):
    import ctypes
    import numpy as np
    import torch
    from skyrmion_solver_b200.core.simulation import Simulation
    from skyrmion_solver_b200.engine import Engine
    from skyrmion_solver_b200.replicas import max_over_ranks

    rank, world, local = dist_env()
    if not torch.cuda.is_available():
        raise RuntimeError("bench.py needs a CUDA device")
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
        pg = dist
    warmup = max(3, args.warmup)
    K = args.steps
    from skyrmion_solver_b200 import _lib
    _lib.call("sky_set_option", 2, 1 if args.staging == "tma" else 0)
    th, p, p_i, p_f = workload_params()
    C, N = int(p_i[5]), int(p_i[6])
    field = workload_field_device(p_i, p_f, dev)

    def barrier():
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize()

    # ---- K timed steps of the resident engine (inputs resident in HBM) ----
    eng = Engine(local)
    iid = eng.add("omega", (p_i, p_f), field, None, precision=FAST)
    stream = torch.cuda.ExternalStream(eng.stream, device=dev)
    eng.step(warmup)
    clocks = ClockSampler(local)
    time.sleep(0.3)
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    clocks.mark_start()
    ev0.record(stream)
    eng.step(K)
    ev1.record(stream)
    ev1.synchronize()
    clocks.mark_end()     # moved to the end of the solves below when they run
    barrier()
    ms = max_over_ranks([ev0.elapsed_time(ev1)], device=dev)[0]   # the job is as slow as its slowest GPU
    ms_step = ms / K
    launches = eng.launches_per_step * K

    # per-launch-kind timing (CUDA events on the engine stream, un-captured launches)
    stages = eng.time_stages(max(5, min(50, K)))
    dom = max(("stage1", "stage2", "stage3", "stage4"), key=lambda k: stages[k])
    alg_bytes = STAGE_PASSES[dom] * C * 4 * N                 # minimal fused schedule: 16 C s per step
    fmt_bytes = stage_passes(dom, FAST) * C * 4 * N           # with the compensated format's extra arrays
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (stages[dom] * 1e-3) / 1e9
    step_bytes = sum(STAGE_PASSES.values()) * C * 4 * N
    traffic = load_traffic(dom)
    eng.close()

    # ---- plain FP64 drop-in path (reference layout, sky_arrested_newton_step), K steps ----
    sim = Simulation(p, th)
    sim.Field.copy_(field)
    sim.Velocity.zero_()
    e = sim.observables()["energy"]
    for _ in range(3):
        e, _ = sim.step(e)
    nplain = max(5, min(50, K))
    torch.cuda.synchronize()
    t0 = torch.cuda.Event(enable_timing=True)
    t1 = torch.cuda.Event(enable_timing=True)
    cur = torch.cuda.current_stream()
    t0.record(cur)
    for _ in range(nplain):
        e, _ = sim.step(e)
    t1.record(cur)
    t1.synchronize()
    plain_ms = max_over_ranks([t0.elapsed_time(t1) / nplain], device=dev)[0]
    del sim

    solve = None
    ref = None
    if not args.quick:
        # ---- the headline: one complete solve through the public API, host buffers in and out ----
        host = torch.empty(C * N, dtype=torch.float64, pin_memory=True)
        host.copy_(field)
        host_np = host.numpy().reshape((C, L, L, L))
        out_pin = torch.empty(C * N, dtype=torch.float64, pin_memory=True)
        out_np = out_pin.numpy().reshape((C, L, L, L))
        barrier()
        tw0 = time.perf_counter()
        ee = Engine(local)
        j = ee.add("omega", (p_i, p_f), host_np, None, precision=FAST)
        t_admit = time.perf_counter() - tw0
        es = torch.cuda.ExternalStream(ee.stream, device=dev)
        st, nsteps, n32, dev_ms, _ = solve_to_tolerance(ee, j, es, args.chunk, args.max_steps)
        tr = time.perf_counter()
        ee._call("sky_engine_read", j, ctypes.c_void_p(out_np.ctypes.data), None, 0)
        t_down = time.perf_counter() - tr
        wall = time.perf_counter() - tw0
        ee.close()
        barrier()
        solve = dict(stats=st, steps=nsteps, fp32_steps=n32, dev_s=dev_ms * 1e-3, wall_s=wall, admit_s=t_admit,
                     download_s=t_down)
        # ---- the plain-FP64 reference solve of the same field (resident FP64 engine) ----
        e64 = Engine(local)
        i64 = e64.add("omega", (p_i, p_f), field, None, precision="fp64")
        s64t = torch.cuda.ExternalStream(e64.stream, device=dev)
        st64, n64, _, dev64_ms, wall64 = solve_to_tolerance(e64, i64, s64t, args.chunk, args.max_steps)
        e64.close()
        ref = dict(stats=st64, steps=n64, dev_s=dev64_ms * 1e-3, wall_s=wall64)
        clocks.mark_end()
    # the reference's own Numba-CUDA run (a child process), after the timed solves
    numba_ref = None
    if not args.quick and not args.no_numba and rank == 0:
        numba_ref = numba_reference_record(field, p, th)

    def ok(r):
        return r is not None and math.isfinite(r["stats"].energy) and r["stats"].gabs <= GRAD_TOL

    value = e2e_value = solve_s = None
    final = None
    if solve is not None:
        dev_s, wall_s = max_over_ranks([solve["dev_s"], solve["wall_s"]], device=dev)
        s = solve["stats"]
        final = {"energy": s.energy, "baryon": s.baryon, "max_abs_gradient": s.gabs, "steps": solve["steps"],
                 "fp32_steps": solve["fp32_steps"], "converged": ok(solve)}
        if ok(ref):
            r = ref["stats"]
            final.update(reference={"schedule": "fp64 engine to max|g| <= %g" % GRAD_TOL, "energy": r.energy,
                                    "baryon": r.baryon, "max_abs_gradient": r.gabs, "steps": ref["steps"]},
                         rel_energy_error=abs(s.energy - r.energy) / abs(r.energy),
                         baryon_error=abs(s.baryon - r.baryon),
                         max_abs_gradient_error=abs(s.gabs - r.gabs))
            final["within_tolerance"] = bool(final["rel_energy_error"] <= REL_ENERGY_TOL and
                                             final["baryon_error"] <= 1e-4 and ok(solve))
        if ok(solve):
            value = world / dev_s
            e2e_value = world / wall_s
            solve_s = wall_s
    plain = {"ms_per_step": plain_ms}
    if ref is not None:
        eng64_dev_s = max_over_ranks([ref["dev_s"]], device=dev)[0]
        plain.update(engine_fp64_solve_s=eng64_dev_s, engine_fp64_steps=ref["steps"],
                     engine_fp64_solves_per_s=world / eng64_dev_s if ok(ref) else None,
                     engine_fp64_ms_per_step=1e3 * eng64_dev_s / ref["steps"],
                     solves_per_s=world / (ref["steps"] * plain_ms * 1e-3) if ok(ref) else None,
                     note="the drop-in path runs the FP64 engine's arithmetic in the reference layout; its "
                          "solve takes the FP64 engine's observed step count at its own timed step rate")
        if value and plain.get("solves_per_s"):
            plain["speedup"] = value / plain["solves_per_s"]
            plain["speedup_vs_engine_fp64"] = value / plain["engine_fp64_solves_per_s"]
    if numba_ref is not None and numba_ref.get("ms_per_step") and ok(ref):
        # the reference's own plain FP64 run takes the FP64 engine's observed step count
        numba_ref["solves_per_s"] = world / (ref["steps"] * numba_ref["ms_per_step"] * 1e-3)
        if value:
            numba_ref["value_over_this"] = value / numba_ref["solves_per_s"]
    field_bytes = C * N * 8
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": warmup,
        "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "theory": "omega (C=5)", "sites": N, "instances_per_gpu": 1,
                   "precision": f"{FAST}: FP32 stencils, compensated hi+lo FP32 field"
                                + (", FP64 defect correction every 16 steps" if FAST == "fp32d" else "")
                                + "; FP64 compensated energy/baryon/arrest; FP64 phase only if the FP32 "
                                  "phase stalls",
                   "dt": DT_FACTOR * H, "couplings": COUPLINGS,
                   "solve": f"arrested Newton flow from the initial field until max|g| <= {GRAD_TOL:g}, "
                            f"checked every {args.chunk} steps; value = 1 / device time of the solve's steps, "
                            "e2e = 1 / wall time of Engine.add (pinned host field) + the steps + per-chunk "
                            "statistics reads + the final field read into pinned host memory",
                   "l2": f"no flush: resident state {9 * C * N * 4 / 1e6:.0f} MB > 126 MB L2",
                   "staging": args.staging, "parallelism": f"replicas x{world}"},
        "latency_s": {"p50": solve_s, "p99": solve_s, "note": "one resident solve per GPU; the serving mode "
                      "(--serve) reports p50/p99 over a request stream"},
        "final": final,
        "steps_rate": {"ms_per_step": ms_step, "site_steps_per_s": world * N * 1e3 / ms_step,
                       "hbm_gbs_step": step_bytes / (ms_step * 1e-3) / 1e9},
        "roofline": {"bound": "hbm", "kernel": f"k_march_stage<Omega,float,{dom[-1]}>"
                     + (" + k_march_defect" if dom == "stage1" and FAST == "fp32d" else ""),
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "traffic": traffic, "algorithmic_bytes_per_launch": alg_bytes,
                     "format_bytes_per_launch": fmt_bytes, "format_achieved": fmt_bytes / (stages[dom] * 1e-3) / 1e9,
                     "issue_active": load_issue_active(dom),
                     "note": "algorithmic bytes: the minimal fused schedule's passes of one C-component FP32 "
                             "field (stage 1: 2, stage 2: 3, stage 3: 4, stage 4: 7); format bytes add the "
                             "compensated field's low parts and the defect correction",
                     "launch_ms": stages[dom], "stage_ms": stages},
        "plain_fp64": plain,
        "reference_numba_cuda": numba_ref,
        "e2e": {"value": e2e_value, "unit": UNIT,
                "h2d_bytes_per_step": field_bytes / solve["steps"] if solve else None,
                "d2h_bytes_per_step": (64 * (solve["steps"] // args.chunk + 1) + field_bytes) / solve["steps"]
                if solve else None,
                "seconds": {"admit": solve["admit_s"], "download": solve["download_s"], "solve": solve["wall_s"]}
                if solve else None},
        "gpu_launches": launches,
        "clocks": clocks.stop(),
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        cb = cpu_baseline()
        nref = ref["steps"] if ok(ref) else None
        cval = cb["site_steps_per_s"] / N / nref if nref else None   # the CPU arm runs the plain FP64 schedule
        line["cpu_baseline"] = {"value": cval, "unit": UNIT, "cores": cb["cores"], "kind": "port",
                                "sample": cb["sample"], "site_steps_per_s": cb["site_steps_per_s"],
                                "steps_per_solve": nref}
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    if rank == 0:
        emit(line)
    return 0


# ---------------------------------------------------------------------------
# calibration: steps to converge, FP64 and FP32 engines
# ---------------------------------------------------------------------------

def run_calibrate(args):
    """Steps to converge: the plain FP64 solve and the mixed schedule the engine serves with.

    fp64:   FP64 engine steps until max|g| <= GRAD_TOL; its final energy is E*.
    mixed:  compensated FP32 until max|g| reaches twice the FP32 gradient floor (or
            stops improving), then FP64 until max|g| <= GRAD_TOL.
    defect: compensated, defect-corrected FP32 until max|g| <= GRAD_TOL (or stalls),
            then FP64 until max|g| <= GRAD_TOL (a check that is short when the
            corrected phase has converged).
    For each, the step after which |E - E*| <= REL_ENERGY_TOL |E*| holds to the end.
    """
    import torch
    from skyrmion_solver_b200.engine import Engine
    from skyrmion_solver_b200.serving import PlateauRule, fp32_gradient_floor
    torch.cuda.set_device(0)
    dev = torch.device("cuda", 0)
    th, p, p_i, p_f = workload_params()
    field = workload_field_device(p_i, p_f, dev)
    chunk = 200
    res = {"workload": WORKLOAD, "chunk": chunk, "grad_tol": GRAD_TOL, "rel_energy_tol": REL_ENERGY_TOL}
    hist = {}
    first = {"fp64": "fp64", "mixed": "fp32c", "defect": "fp32d"}
    for sched in ("fp64", "mixed", "defect"):
        eng = Engine(0)
        prec = first[sched]
        iid = eng.add("omega", (p_i, p_f), field, None, precision=prec)
        # the defect-corrected phase can go to the tolerance itself; the plain FP32 phase stops near its floor
        rule = PlateauRule(GRAD_TOL if sched == "defect" else 2.0 * fp32_gradient_floor(p_f))
        switch = None
        h = [(0, eng.stats(iid).energy, float("inf"), prec)]
        t0 = time.perf_counter()
        n = 0
        while n < args.max_steps:
            eng.step(chunk)
            n += chunk
            st = eng.stats(iid)
            h.append((n, st.energy, st.gabs, prec))
            if not math.isfinite(st.energy):
                break
            if prec == "fp64":
                if st.gabs <= GRAD_TOL:
                    break
            elif rule.update(st.gabs, chunk):
                eng.set_precision(iid, "fp64")
                prec = "fp64"
                switch = n
        secs = time.perf_counter() - t0
        eng.close()
        hist[sched] = h
        res[f"{sched}_total_steps"] = n
        res[f"{sched}_switch_step"] = switch
        res[f"{sched}_seconds"] = secs
        res[f"{sched}_final_energy"] = h[-1][1]
        res[f"{sched}_final_max_abs_gradient"] = h[-1][2]
        print(json.dumps({"schedule": sched, "steps": n, "switch": switch, "secs": secs, "E": h[-1][1],
                          "gabs": h[-1][2]}), flush=True)
    e_star = res["fp64_final_energy"]
    res["reference_energy"] = e_star

    def settle(hh):
        """First recorded step after which |E - E*| <= tol |E*| holds to the end of the run."""
        s = None
        for n, e, _, _ in hh:
            if abs(e - e_star) <= REL_ENERGY_TOL * abs(e_star):
                if s is None:
                    s = n
            else:
                s = None
        return s

    for sched in ("fp64", "mixed", "defect"):
        s = settle(hist[sched])
        res[f"{sched}_steps_to_converge"] = s
        res[f"{sched}_final_rel_energy_error"] = abs(res[f"{sched}_final_energy"] - e_star) / abs(e_star)
        if sched == "fp64":
            continue
        sw = res[f"{sched}_switch_step"]
        if s is not None:
            res[f"{sched}_fp32_steps"] = min(s, sw) if sw is not None else s
            res[f"{sched}_fp64_steps"] = max(0, s - sw) if sw is not None else 0
    res["fp64_reached_grad_tol"] = res["fp64_final_max_abs_gradient"] <= GRAD_TOL
    res["history_every"] = chunk * 10
    for sched in ("fp64", "mixed", "defect"):
        res[f"{sched}_history"] = hist[sched][::10]
    res["command"] = "python bench.py --calibrate"
    os.makedirs(os.path.dirname(CALIBRATION), exist_ok=True)
    out = args.out or CALIBRATION
    with open(out, "w") as fh:
        json.dump(res, fh, indent=1)
    print(json.dumps({k: v for k, v in res.items() if "history" not in k}), flush=True)
    return 0


# ---------------------------------------------------------------------------
# serving: a Poisson request stream, continuous batching vs serial plain FP64
# ---------------------------------------------------------------------------

SERVE_THEORIES = {"nuclear": {}, "omega": dict(COUPLINGS),
                  "coulomb": dict(f_pi=105.9, m_pi=138.0, g=4.010, e=0.302822),
                  "rho": dict(mpi=0.586, mrho=3.29, c_alpha=0.2256)}


def serve_requests(n, rate, seed, mix, bmax, max_side, tol, max_steps):
    """Requests drawn as the serving configuration draws them: theory by weight, B uniform in 1..bmax,
    side min(max_side, max(48, ceil((48 + 12 B) / 16) * 16)), h = 0.2, dt = 0.2 h (rho: h = 0.05, on
    which its B=1 soliton survives relaxation, and dt = 0.05 h), a product of B hedgehogs at seeded
    positions (minimum separation 2) with Haar-random orientations."""
    import numpy as np
    from skyrmion_solver_b200 import theories as T
    from skyrmion_solver_b200.serving import Request, poisson_arrivals
    rng = np.random.default_rng(seed)
    names = list(mix)
    w = np.array([mix[k] for k in names], dtype=np.float64)
    w /= w.sum()
    arrivals = poisson_arrivals(rate, n, seed)
    reqs = []
    for k in range(n):
        name = names[int(rng.choice(len(names), p=w))]
        B = int(rng.integers(1, bmax + 1))
        side = int(min(max_side, max(48, math.ceil((48 + 12 * B) / 16) * 16)))
        h = 0.05 if name == "rho" else 0.2      # rho unwinds to the vacuum on coarser lattices
        th = T.by_short_name(name)
        prm = th.params.default_params(xlen=side, ylen=side, zlen=side, lsx=h, lsy=h, lsz=h, xsize=h * (side - 1),
                                       ysize=h * (side - 1), zsize=h * (side - 1),
                                       time_step=(0.05 if name == "rho" else 0.2) * h, **SERVE_THEORIES[name])
        p_i, p_f = th.params.pack_device_params(prm.resolved())
        p_i = np.asarray(p_i, np.int32)
        p_f = np.asarray(p_f, np.float64)
        cfg = {"mode": "cloud", "count": B, "seed": seed * 1000 + k, "scale": 1.5, "vacuum_shell": 2}
        # the field is built on the device when the request is admitted (sky_init_field)
        reqs.append((Request(k, name, p_i, p_f, None, float(arrivals[k]), tol, max_steps, init=cfg), prm, th))
    return reqs


def run_serve(args):
    """The serving stream on N GPUs (torchrun for N > 1): every rank draws the same request
    list and serves its share (replicas.partition: least work so far, in arrival order) on
    its own engine; no data crosses GPUs.  The serial plain FP64 baseline solves each rank's
    share one request after another on that rank's GPU.  Rank 0 merges and prints."""
    import numpy as np
    import torch
    from skyrmion_solver_b200.core.simulation import Simulation
    from skyrmion_solver_b200.engine import Engine
    from skyrmion_solver_b200.replicas import gather_objects, max_over_ranks, merge_served, partition
    from skyrmion_solver_b200.serving import Server
    from skyrmion_solver_b200.theories._init_common import build_device_field, seed_omega
    rank, world, local = dist_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=dev)
    mix = dict(kv.split(":") for kv in args.mix.split(","))
    mix = {k: float(v) for k, v in mix.items()}
    reqs = serve_requests(args.requests, args.rate, args.seed, mix, args.bmax, args.max_side, GRAD_TOL,
                          args.max_steps)
    mine = {r.rid for r in partition([r for r, _, _ in reqs], world)[rank]}
    my_reqs = [x for x in reqs if x[0].rid in mine]

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    # 1. continuous batching on the resident engine
    barrier()
    with Engine(local) as eng:
        srv = Server(eng, chunk=64, fp32_mode=args.schedule, defect_period=args.defect_period,
                     switch_factor=args.switch_factor, plateau_chunks=args.plateau_chunks)
        for r, _, _ in my_reqs:
            srv.submit(r)
        torch.cuda.synchronize()
        served = {x.rid: x for x in srv.run()}
    barrier()
    # 2. the same requests solved one after another on the plain FP64 drop-in path
    serial = {}
    t_all = 0.0
    for r, prm, th in ([] if args.no_serial else my_reqs):
        sim = Simulation(prm, th)
        f0 = build_device_field(r.theory, r.p_i, r.p_f, r.init, device=local)   # the field the server built
        if r.theory == "omega":
            seed_omega(f0, r.p_i, r.p_f)
        sim.Field.copy_(f0)
        sim.Velocity.zero_()
        e = sim.observables()["energy"]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        n, status = 0, "not_converged"
        while n < args.max_steps:
            e, _ = sim.step(e)
            n += 1
            if n % 64 == 0:
                if not math.isfinite(e):
                    status = "failed"
                    break
                if float(sim.EnergyGradient.abs().max()) <= GRAD_TOL:
                    status = "converged"
                    break
        torch.cuda.synchronize()
        dt = time.perf_counter() - t0
        t_all += dt
        serial[r.rid] = dict(status=status, steps=n, energy=e, seconds=dt)
        del sim
    if args.no_serial:
        serial = {k: dict(status=None, steps=None, energy=math.nan, seconds=None) for k in served}
    # merge over ranks
    theory_of = {r.rid: r.theory for r, _, _ in reqs}
    rows = [(k, served[k].status, served[k].latency, served[k].finished) for k in sorted(served)]
    summ = merge_served(gather_objects(rows))
    summ["batch_steps_per_rank"] = max_over_ranks([srv.steps_run], device=dev)[0]
    per_request = [dict(rid=k, theory=theory_of[k], sites=int(reqs[k][0].p_i[6]), rank=rank,
                        energy=served[k].energy, baryon=served[k].baryon, serial_energy=serial[k]["energy"],
                        served_steps=served[k].steps, fp32_steps=served[k].fp32_steps,
                        latency_s=served[k].latency, status=served[k].status,
                        serial_status=serial[k]["status"], serial_steps=serial[k]["steps"],
                        serial_s=serial[k]["seconds"]) for k in sorted(served)]
    per_request = sorted((d for part in gather_objects(per_request) for d in part), key=lambda d: d["rid"])
    serial_wall = max_over_ranks([t_all], device=dev)[0]     # the ranks' serial solves run side by side
    if world > 1:
        torch.distributed.destroy_process_group()
    if rank != 0:
        return 0
    # relative to max(|E|, 1): a configuration that unwinds to the vacuum (E -> 0) compares absolutely
    rel = [abs(d["energy"] - d["serial_energy"]) / max(abs(d["serial_energy"]), 1.0) for d in per_request
           if d["status"] == "converged" and d["serial_status"] == "converged"]
    n_serial = sum(d["serial_status"] == "converged" for d in per_request)
    serial_sps = n_serial / serial_wall if serial_wall > 0 else None
    # per theory: counts by outcome and time-to-converged percentiles, served and serial
    by_theory = {}
    for th_name in sorted(set(theory_of.values())):
        ds = [d for d in per_request if d["theory"] == th_name]
        lat = np.array([d["latency_s"] for d in ds if d["status"] == "converged"])
        by_theory[th_name] = {
            "requests": len(ds),
            "served": {st: sum(d["status"] == st for d in ds) for st in ("converged", "failed", "not_converged")},
            "serial": {st: sum(d["serial_status"] == st for d in ds) for st in ("converged", "failed",
                                                                                 "not_converged")},
            "p50_s": float(np.percentile(lat, 50)) if lat.size else None,
            "p99_s": float(np.percentile(lat, 99)) if lat.size else None}
    line = {"mode": "serve", "metric": METRIC, "unit": UNIT, "n_gpus": world,
            "config": {"workload": "poisson_stream", "requests": args.requests, "rate_per_s": args.rate,
                       "mix": mix, "B": f"1..{args.bmax}", "max_side": args.max_side,
                       "h": "0.2 (rho 0.05)", "dt": "0.2 h (rho 0.05 h)",
                       "tol_max_abs_gradient": GRAD_TOL, "defect_period": args.defect_period or 16,
                       "routing": "replicas.partition (least work first, arrival order)" if world > 1 else None,
                       "schedule": {"fp64": "fp64 throughout",
                                    "fp32d": "fp32d until max|g| <= tol or a stall, then fp64"}.get(
                           args.schedule, f"{args.schedule} until {args.switch_factor:g} x the FP32 gradient "
                                          f"floor or a stall of {args.plateau_chunks * 64} steps, then fp64")},
            "served": summ,
            "by_theory": by_theory,
            "serial_plain_fp64": None if args.no_serial else {"converged": n_serial, "seconds": serial_wall,
                                                              "solves_per_s": serial_sps},
            "speedup_solves_per_s": (summ["solves_per_s"] / serial_sps) if (summ["solves_per_s"] and serial_sps)
            else None,
            "max_rel_energy_diff_vs_plain_fp64": max(rel) if rel else None,
            "per_request": per_request}
    emit(line)
    return 0


# ---------------------------------------------------------------------------
# batched relaxation (48 instances of mixed theory and size in one engine)
# ---------------------------------------------------------------------------

def run_batch(args):
    """Throughput of one engine holding a batch like the batched-relaxation configuration:
    B uniform in 1..8, side ceil((48 + 12 B) / 16) * 16, h = 0.2, pion or rho (50/50), seeded product
    ansatz of B hedgehogs, compensated FP32; every instance advances in the same launches."""
    import numpy as np
    import torch
    from skyrmion_solver_b200.engine import Engine
    from skyrmion_solver_b200 import theories as T
    from skyrmion_solver_b200.theories._init_common import build_host_field
    torch.cuda.set_device(0)
    rng = np.random.default_rng(args.seed)
    eng = Engine(0)
    sites = {"nuclear": 0, "rho": 0}
    comps = 0
    members = {}
    for k in range(args.instances):
        name = "nuclear" if rng.random() < 0.5 else "rho"
        B = int(rng.integers(1, 9))
        side = int(math.ceil((48 + 12 * B) / 16) * 16)
        h = 0.2
        th = T.by_short_name(name)
        dt = 0.2 * h if name == "nuclear" else 0.05 * h
        prm = th.params.default_params(xlen=side, ylen=side, zlen=side, lsx=h, lsy=h, lsz=h, xsize=h * (side - 1),
                                       ysize=h * (side - 1), zsize=h * (side - 1), time_step=dt,
                                       **SERVE_THEORIES[name])
        p_i, p_f = th.params.pack_device_params(prm.resolved())
        p_i, p_f = np.asarray(p_i, np.int32), np.asarray(p_f, np.float64)
        f = build_host_field(name, p_i, p_f, {"mode": "cloud", "count": B, "seed": 100 + k, "scale": 1.5,
                                                "vacuum_shell": 2})
        members[eng.add(name, (p_i, p_f), f, None, precision=FAST)] = (name, p_i, p_f)
        sites[name] += side ** 3
        comps += int(p_i[5]) * side ** 3
    N = sites["nuclear"] + sites["rho"]
    warmup = max(3, args.warmup)
    K = args.steps
    stream = torch.cuda.ExternalStream(eng.stream)

    def timed():
        eng.step(warmup)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        eng.step(K)
        b.record(stream)
        b.synchronize()
        return a.elapsed_time(b) / K

    ms = timed()
    tuned = None
    if args.tune:
        # the autotuner's (staging, x-chunk) per lattice shape, measured on probe instances
        # (untimed), then applied to every instance of the batch in place
        from skyrmion_solver_b200 import autotune
        cache = autotune.TuneCache(None)
        choices = {}
        default = {iid: (eng.staging(iid), eng.xc(iid)) for iid in members}
        for iid, (name, p_i, p_f) in members.items():
            res = autotune.tune(name, p_i, p_f, FAST, cache=cache, steps=6)
            autotune.apply(eng, iid, name, FAST, p_i, cache)
            choices[f"{name} {int(p_i[0])}^3"] = {k: res[k] for k in ("xc", "tma", "pair")}
        ms_tuned = timed()
        # the flow has moved on (arrested steps are cheaper): time the defaults again, now
        for iid, (st, xc) in default.items():
            eng.set_staging(iid, *st)
            eng.retile(iid, xc)
        ms_default_after = timed()
        # batch-aware chunking: a full batch fills the GPU with tiles anyway, so whole-lattice
        # x-chunks (fewest halo re-reads) may beat the per-shape choice made for an instance alone
        for iid, (name, p_i, p_f) in members.items():
            eng.retile(iid, int(p_i[0]))
        tuned = {"ms_per_step": ms_tuned, "defaults_ms_per_step_after": ms_default_after,
                 "whole_lattice_chunks_ms_per_step": timed(), "choices": choices}
    stages = eng.time_stages(max(3, min(20, K)))
    stats = eng.stats_all()
    finite = sum(math.isfinite(st.energy) for st in stats.values())
    emit({"mode": "batch", "instances": args.instances, "sites": N, "sites_by_theory": sites,
          "field_values": comps, "device_bytes": eng.bytes, "ms_per_step": ms,
          "site_steps_per_s": N / (ms * 1e-3), "algorithmic_gbs": 18 * 4 * comps / (ms * 1e-3) / 1e9,
          "stage_ms": stages, "finite_instances": finite, "launches_per_step": eng.launches_per_step,
          "precision": FAST, "dt": {"nuclear": "0.2 h", "rho": "0.05 h"}, "tuned": tuned})
    eng.close()
    return 0


# ---------------------------------------------------------------------------
# RK4 dynamics: two boosted B=2 tori, Coulomb variant, energy audit
# ---------------------------------------------------------------------------

def run_dynamics(args):
    """Two B=2 toroidal (z^2 rational map) skyrmions at x = -/+3, the second isorotated by a seeded
    Haar-random SU(2) element, combined by quaternion product, boosted toward each other at relative
    velocity 0.3 (V = -u(x) d_x phi projected orthogonal to phi, u = 0.15 tanh(-x)), Coulomb variant
    (or --theory), side^3 sites with h = 0.15 (or --h), dt = 0.1 h, killkinen = 0 (RK4 dynamics), compensated
    FP32 (or --precision).  Every 50 steps the FP64 energy audit (sky_engine_audit) evaluates the
    potential Phi that the kernels integrate and K = (1/2) h^3 sum_c s_c |V_c|^2; H = Phi + K."""
    import numpy as np
    import torch
    from skyrmion_solver_b200.engine import Engine
    from skyrmion_solver_b200 import initial as ini
    from skyrmion_solver_b200 import theories as T
    torch.cuda.set_device(0)
    L, h = args.side, args.h
    name = args.theory
    th = T.by_short_name(name)
    prm = th.params.default_params(xlen=L, ylen=L, zlen=L, lsx=h, lsy=h, lsz=h, xsize=h * (L - 1),
                                   ysize=h * (L - 1), zsize=h * (L - 1), time_step=0.1 * h, killkinen=False,
                                   **SERVE_THEORIES[name])
    p_i, p_f = th.params.pack_device_params(prm.resolved())
    p_i, p_f = np.asarray(p_i, np.int32), np.asarray(p_f, np.float64)
    rng = np.random.default_rng(args.seed)
    dims = (L, L, L)
    prof = ini.exp_profile(1.5)
    left = ini.rational_map(dims, (h, h, h), 2, prof, center=(-3.0, 0.0, 0.0))
    right = ini.isorotate(ini.rational_map(dims, (h, h, h), 2, prof, center=(3.0, 0.0, 0.0)), ini.haar_su2(rng))
    phi = ini.normalise(ini.quat_mul(left, right))
    x = ini.coords(dims, (h, h, h))[0]
    dphi = np.gradient(phi, h, axis=1)
    V = -(0.15 * np.tanh(-x))[None] * dphi
    V -= (V * phi).sum(axis=0) * phi
    C = int(p_i[5])
    F = ini.with_extra_components(phi, C)
    Vf = ini.with_extra_components(V, C)
    ini.vacuum_shell(F, 2)
    Vf[:, :2] = Vf[:, -2:] = 0.0
    Vf[:, :, :2] = Vf[:, :, -2:] = 0.0
    Vf[:, :, :, :2] = Vf[:, :, :, -2:] = 0.0
    with Engine(0) as eng:
        i = eng.add(name, (p_i, p_f), F, Vf, precision=args.precision)
        audit = []

        def record(n):
            st = eng.stats(i)
            a = eng.audit(i)
            audit.append((n, a["potential"], a["kinetic"], st.energy, st.baryon))

        record(0)
        stream = torch.cuda.ExternalStream(eng.stream)
        torch.cuda.synchronize()
        t_dev = t_audit = 0.0
        for n in range(50, args.steps + 1, 50):
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            eng.step(50)
            b.record(stream)
            b.synchronize()
            t_dev += a.elapsed_time(b)
            t0 = time.perf_counter()
            record(n)
            t_audit += time.perf_counter() - t0
    H = [phi + k for _, phi, k, _, _ in audit]
    drift = [abs(v - H[0]) / abs(H[0]) for v in H]
    emit({"mode": "dynamics", "theory": name, "sites": L ** 3, "h": h, "dt": 0.1 * h, "steps": args.steps,
          "ms_per_step": t_dev / args.steps,
          "site_steps_per_s": L ** 3 * args.steps / (t_dev * 1e-3), "precision": args.precision,
          "audit_ms": 1e3 * t_audit / max(1, len(audit) - 1),
          "H0": H[0], "H_final": H[-1], "max_rel_H_drift": max(drift),
          "baryon": [audit[0][4], audit[-1][4]],
          "audit_every_50": [dict(step=n, Phi=phi, K=k, E_coded=e) for n, phi, k, e, _ in
                             audit[:: max(1, len(audit) // 20)]],
          "note": "H = Phi + K from sky_engine_audit (FP64): Phi is the potential whose (anti-)gradient the "
                  "kernels integrate, K the kinetic term with the auxiliary field's negative sign (omega, "
                  "Coulomb); E_coded is the variant's coded energy (reference compute_energy)"})
    return 0


def run_render(args):
    """The headless viewer on a side^3 nuclear lattice (h = 0.1) holding the reference's
    smorgasbord of 8 rational-map lumps: the RGBA volume builder (min / max, then the
    transposing fill; 48 algorithmic bytes per site: the density read by both passes, three
    pion components, one float4 written) and the 1200 x 900 ray-march of the default view in both colourings, each timed
    with CUDA events over --steps calls after --warmup.  Inputs (side 192: 340 MB) exceed L2."""
    import numpy as np
    import torch
    from skyrmion_solver_b200 import theories as T
    from skyrmion_solver_b200.core.simulation import Simulation
    from skyrmion_solver_b200.visualization import HeadlessRenderer
    torch.cuda.set_device(0)
    L = args.side
    th = T.by_short_name("nuclear")
    prm = th.params.default_params(xlen=L, ylen=L, zlen=L, lsx=0.1, lsy=0.1, lsz=0.1, xsize=0.1 * (L - 1),
                                   ysize=0.1 * (L - 1), zsize=0.1 * (L - 1))
    sim = Simulation(prm, th)
    sim.initialize({"mode": "smorgasbord", "count": 8, "seed": 0})
    sim.compute_baryon_density()
    r = HeadlessRenderer(1200, 900, L)
    r.bind_sim(sim)
    peak, peak_src = measured_peaks()
    clocks = ClockSampler(0)

    def timed(fn):
        for _ in range(max(args.warmup, 1)):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / args.steps

    clocks.mark_start()
    t_vol = timed(lambda: r.build_volume(sim.en, sim.Field))
    r.set_display_mode(1)
    t_tf = timed(r.draw)
    r.set_display_mode(2)
    t_pion = timed(r.draw)
    clocks.mark_end()
    clk = clocks.stop()
    N = L ** 3
    achieved = 48.0 * N / (t_vol * 1e-3) / 1e9
    img = r.image.cpu().numpy()
    emit({"mode": "render", "sites": N, "data": "synthetic: the reference's smorgasbord initial field",
          "volume": {"ms": t_vol, "bytes_per_site": 48, "achieved_gbs": achieved, "peak_gbs": peak,
                     "peak_source": peak_src, "frac": achieved / peak, "extrema": list(r.extrema)},
          "render": {"width": 1200, "height": 900, "ms": {"transfer": t_tf, "pion": t_pion},
                     "frames_per_s": {"transfer": 1e3 / t_tf, "pion": 1e3 / t_pion},
                     "covered_pixels": float((img[..., :3] != 1.0).any(-1).mean())},
          "steps": args.steps, "warmup": args.warmup, "clocks": clk})


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=("ours", "reference"), default="ours")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--quick", action="store_true", help="skip the two timed solves (K-step rate only)")
    ap.add_argument("--no-numba", action="store_true", help="skip the reference's Numba-CUDA run")
    ap.add_argument("--numba-reference", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--field", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--chunk", type=int, default=128, help="steps between convergence checks of a solve")
    ap.add_argument("--staging", choices=("tma", "cp.async"), default="tma",
                    help="how the engine's stage kernels stage lattice planes in shared memory")
    ap.add_argument("--calibrate", action="store_true")
    ap.add_argument("--max-steps", type=int, default=240000)
    ap.add_argument("--out", default=None)
    ap.add_argument("--serve", action="store_true", help="serving stream: continuous batching vs serial plain FP64")
    ap.add_argument("--requests", type=int, default=24)
    ap.add_argument("--rate", type=float, default=20.0)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--mix", default="nuclear:0.4,omega:0.3,rho:0.2,coulomb:0.1",
                    help="serving: theory weights (the serving stream's mix by default)")
    ap.add_argument("--bmax", type=int, default=12, help="serving: baryon numbers drawn from 1..bmax")
    ap.add_argument("--schedule", choices=("fp32d", "fp32c", "fp32", "fp64"), default="fp64",
                    help="serving precision schedule: FP32 phase then FP64, or FP64 throughout")
    ap.add_argument("--max-side", type=int, default=192)
    ap.add_argument("--switch-factor", type=float, default=2.0,
                    help="serving: fp32 / fp32c requests switch to FP64 at this multiple of the FP32 gradient floor")
    ap.add_argument("--plateau-chunks", type=int, default=256,
                    help="serving: 64-step chunks without a 1%% gain in max|g| after which the FP32 phase ends")
    ap.add_argument("--no-serial", action="store_true", help="serving: skip the serial plain FP64 solves")
    ap.add_argument("--defect-period", type=int, default=None,
                    help="serving: steps between refreshes of the fp32d correction (default 16)")
    ap.add_argument("--render", action="store_true", help="headless viewer: volume builder and ray-march")
    ap.add_argument("--batch", action="store_true", help="48 mixed pion / rho instances in one engine")
    ap.add_argument("--instances", type=int, default=48)
    ap.add_argument("--tune", action="store_true", help="batch: also time the batch with autotuned staging and chunks")
    ap.add_argument("--dynamics", action="store_true", help="RK4 dynamics of two boosted tori with energy audit")
    ap.add_argument("--side", type=int, default=192)
    ap.add_argument("--theory", choices=("coulomb", "nuclear", "omega"), default="coulomb",
                    help="dynamics: theory variant")
    ap.add_argument("--h", type=float, default=0.15, help="dynamics: lattice spacing (dt = 0.1 h)")
    ap.add_argument("--precision", choices=("fp32c", "fp32", "fp32d", "fp64"), default="fp32c",
                    help="dynamics: engine precision")
    args = ap.parse_args()
    if args.render:
        return run_render(args)
    if args.batch:
        return run_batch(args)
    if args.dynamics:
        if args.steps == 2000:
            args.steps = 5000
        return run_dynamics(args)
    if args.calibrate:
        return run_calibrate(args)
    if args.serve:
        if args.max_steps == 240000:
            args.max_steps = 20000
        return run_serve(args)
    if args.numba_reference:
        return run_numba_reference(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
