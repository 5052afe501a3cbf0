"""Resident batched engine: many lattice instances advanced together on one GPU.

The engine (``sky_engine_*`` in the C ABI) keeps each instance's field,
velocity and RK4 slopes resident in HBM, runs the arrested-Newton step of
skyrmion_solver ``core/integrator.py:284-410`` as fused stage kernels over all
instances of a theory at once, reduces energies and baryon numbers in FP64
with compensated summation, takes the arrest decision on the device and
replays the per-step launches from a CUDA graph.  Instances are FP32
(``precision="fp32"``, stage arithmetic and state in FP32), FP32 with a
compensated field (``"fp32c"``: the field is an unevaluated FP32 sum hi + lo
updated in FP64, so sub-ulp updates near convergence are not lost), FP32 with a
compensated field and a defect-corrected gradient (``"fp32d"``: every 16 steps the
FP64 gradient of the field is evaluated and its difference to the FP32 one is
added to the FP32 stage gradients, so the solve converges to the FP64 fixed
point at FP32 cost) or FP64.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import THEORY_IDS, f64p, i32p

PRECISIONS = {"fp32": 0, "fp64": 1, "fp32c": 2, "fp32d": 3}
PRECISION_NAMES = {v: k for k, v in PRECISIONS.items()}


@dataclass
class StepStats:
    energy: float
    baryon: float
    err: float        # signed max of the stage-4 gradient (the reference's err)
    gabs: float       # max |gradient| of that stage
    arrested: bool    # velocity zeroed for the next step
    step: int
    precision: str = ""
    kinetic: float = 0.0   # (1/2) h^3 sum |V'|^2 after the step (before any arrest)


def _theory_id(theory) -> int:
    if isinstance(theory, int):
        return theory
    t = getattr(theory, "SHORT_NAME", theory)
    if t not in THEORY_IDS:
        raise ValueError(f"unknown theory {theory!r}")
    return THEORY_IDS[t]


def _packed(params, theory=None):
    """(p_i, p_f) from a Params / ResolvedParams object or a (p_i, p_f) pair."""
    if isinstance(params, tuple) and len(params) == 2:
        p_i, p_f = params
    else:
        rp = params.resolved() if hasattr(params, "resolved") else params
        if theory is None or not hasattr(theory, "params"):
            raise ValueError("pass the theory module with Params objects")
        p_i, p_f = theory.params.pack_device_params(rp)
    return np.ascontiguousarray(p_i, dtype=np.int32), np.ascontiguousarray(p_f, dtype=np.float64)


class Engine:
    def __init__(self, device: int = 0):
        lib = _lib.load()
        h = ctypes.c_void_p()
        _lib.check(lib.sky_engine_create(int(device), ctypes.byref(h)), "sky_engine_create")
        self._h = h
        self._lib = lib
        self.device = device
        self.meta = {}

    # ------------------------------------------------------------------
    def close(self):
        if self._h:
            self._lib.sky_engine_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _call(self, name, *args):
        _lib.check(getattr(self._lib, name)(self._h, *args), name)

    # ------------------------------------------------------------------
    def add(self, theory, params, field, velocity=None, precision: str = "fp32") -> int:
        """Admit an instance; field / velocity: FP64 arrays (host numpy or CUDA tensors) of shape (C, X, Y, Z)."""
        tid = _theory_id(theory)
        p_i, p_f = _packed(params, theory)
        on_dev = 0
        keep = []

        def ptr(a):
            nonlocal on_dev
            if a is None:
                return None
            try:
                import torch
                if isinstance(a, torch.Tensor) and a.is_cuda:
                    if a.device.index != self.device:
                        raise ValueError(f"device tensor on {a.device}, but the engine runs on cuda:{self.device}")
                    on_dev = 1
                    t = a.detach().to(torch.float64).contiguous()
                    keep.append(t)
                    return ctypes.c_void_p(t.data_ptr())
            except ImportError:  # pragma: no cover
                pass
            h = np.ascontiguousarray(np.asarray(a, dtype=np.float64))
            keep.append(h)
            return ctypes.c_void_p(h.ctypes.data)

        fp = ptr(field)
        vp = ptr(velocity)
        if velocity is not None and on_dev != (1 if not isinstance(keep[-1], np.ndarray) else 0):
            raise ValueError("field and velocity must both be host arrays or both device tensors")
        if on_dev:
            # the engine reads device inputs on its own stream: finish torch's pending work first
            import torch
            torch.cuda.current_stream(torch.device("cuda", self.device)).synchronize()
        C = int(p_i[5])
        n = C * int(p_i[6])
        if (keep[0].numel() if hasattr(keep[0], "numel") else keep[0].size) != n:
            raise ValueError(f"field has {keep[0].size} values, expected C*N = {n}")
        out = ctypes.c_int(-1)
        self._call("sky_engine_add", tid, i32p(p_i), len(p_i), f64p(p_f), len(p_f), PRECISIONS[precision], fp, vp,
                   on_dev, ctypes.byref(out))
        iid = int(out.value)
        self.meta[iid] = dict(theory=tid, p_i=p_i, p_f=p_f, C=C, dims=tuple(int(v) for v in p_i[:3]),
                              precision=precision)
        return iid

    def remove(self, iid: int):
        self._call("sky_engine_remove", int(iid))
        self.meta.pop(iid, None)

    def set_precision(self, iid: int, precision: str):
        self._call("sky_engine_set_precision", int(iid), PRECISIONS[precision])
        self.meta[iid]["precision"] = precision

    def retile(self, iid: int, xc: int = 0):
        """x-chunk of the marching kernels for this instance (0 = automatic)."""
        self._call("sky_engine_retile", int(iid), int(xc))

    def set_staging(self, iid: int, tma: bool, pair: bool = False):
        """Plane staging of this instance: TMA box copies or cp.async, and z-pair tiles."""
        self._call("sky_engine_set_staging", int(iid), int(bool(tma)), int(bool(pair)))

    def staging(self, iid: int) -> tuple:
        """(tma, pair) of this instance."""
        t, q = ctypes.c_int(0), ctypes.c_int(0)
        self._call("sky_engine_get_staging", int(iid), ctypes.byref(t), ctypes.byref(q))
        return bool(t.value), bool(q.value)

    def set_defect_period(self, iid: int, period: int):
        """Steps between refreshes of an fp32d instance's FP64 correction (default 16)."""
        self._call("sky_engine_set_defect_period", int(iid), int(period))

    def xc(self, iid: int) -> int:
        return int(self._lib.sky_engine_get_xc(self._h, int(iid)))

    def audit(self, iid: int) -> dict:
        """FP64 energy audit of the RK4 dynamics of `iid`'s current state: the potential
        `potential` whose (anti-)gradient the kernels integrate, the signed kinetic term
        `kinetic` and their sum `hamiltonian` (conserved up to the O(h^4) stencil gap)."""
        out = np.zeros(2)
        self._call("sky_engine_audit", int(iid), f64p(out))
        return {"potential": float(out[0]), "kinetic": float(out[1]), "hamiltonian": float(out[0] + out[1])}

    def set_active(self, iid: int, active: bool):
        self._call("sky_engine_set_active", int(iid), 1 if active else 0)

    def step(self, nsteps: int = 1):
        self._call("sky_engine_step", int(nsteps))

    def synchronize(self):
        self._call("sky_engine_synchronize")

    @property
    def stream(self) -> int:
        return int(self._lib.sky_engine_stream(self._h) or 0)

    def stats(self, iid: int, step: int = -1) -> StepStats:
        out = (ctypes.c_double * 8)()
        self._call("sky_engine_stats_ex", int(iid), int(step), out)
        return StepStats(out[0], out[1], out[2], out[3], bool(out[4]), int(out[5]),
                         PRECISION_NAMES.get(int(out[7]), ""), out[6])

    def stats_all(self) -> dict:
        cap = max(1, len(self.meta))
        ids = (ctypes.c_int * cap)()
        vals = (ctypes.c_double * (7 * cap))()
        cnt = ctypes.c_int(0)
        self._call("sky_engine_stats_all", ids, vals, cap, ctypes.byref(cnt))
        res = {}
        for k in range(cnt.value):
            o = vals[7 * k:7 * k + 7]
            res[int(ids[k])] = StepStats(o[0], o[1], o[2], o[3], bool(o[4]), int(o[5]),
                                         PRECISION_NAMES.get(int(o[6]), "fp32"))
        return res

    def read(self, iid: int, velocity: bool = True):
        """(field, velocity) as FP64 numpy arrays of shape (C, X, Y, Z)."""
        m = self.meta[iid]
        shape = (m["C"],) + m["dims"]
        f = np.empty(shape)
        v = np.empty(shape) if velocity else None
        self._call("sky_engine_read", int(iid), ctypes.c_void_p(f.ctypes.data),
                   ctypes.c_void_p(v.ctypes.data) if v is not None else None, 0)
        return f, v

    def read_device(self, iid: int, field_out, velocity_out=None):
        """Copy the state into FP64 CUDA tensors (reference layout) without a host round trip."""
        self._call("sky_engine_read", int(iid), _lib.dptr(field_out),
                   _lib.dptr(velocity_out) if velocity_out is not None else None, 1)

    def view(self, iid: int, density: str = "baryon"):
        """The FP64 buffers a renderer reads, materialised on the device from an instance of any
        precision: the reference's ``sim.Field`` (reference layout, C*N values) and ``sim.en``
        after ``compute_baryon_density()`` (b h^3 per site) or the energy kernel (e h^3), as read
        by th/nuclear_skyrme/render_gl.py:157-222.  Returns (field, en) CUDA tensors; nothing
        passes through the host."""
        import torch
        if density not in ("baryon", "energy"):
            raise ValueError("density must be 'baryon' or 'energy'")
        m = self.meta[iid]
        N = int(m["p_i"][6])
        dev = torch.device("cuda", self.device)
        # the C functions launch on the current device: make the engine's device current
        with torch.cuda.device(dev):
            stream = torch.cuda.current_stream(dev)
            field = torch.empty(m["C"] * N, dtype=torch.float64, device=dev)
            stream.synchronize()                           # the engine writes on its own stream
            self.read_device(iid, field)                   # synchronous on the engine's stream
            en = torch.zeros(N, dtype=torch.float64, device=dev)
            fn = "sky_baryon_density" if density == "baryon" else "sky_energy_density"
            _lib.call(fn, m["theory"], i32p(m["p_i"]), len(m["p_i"]), f64p(m["p_f"]), len(m["p_f"]), _lib.dptr(en),
                      _lib.dptr(field), _lib.stream_ptr(stream))
        return field, en

    def diagnostics(self, iid: int) -> dict:
        """Centre of mass and RMS radius of an instance of any precision and, for the nuclear
        model, its U, V and W inertia tensors, quadrupole tensor and D-term: the fused FP64
        passes behind Simulation.compute_center_of_mass ... compute_D_term
        (th/nuclear_skyrme/observables.py:182-487), run on the instance's FP64 field."""
        import math
        import numpy as np
        import torch
        from .core import observables as ob
        m = self.meta[iid]
        p_i, p_f = m["p_i"], m["p_f"]
        dev = torch.device("cuda", self.device)
        # the C functions launch on the current device and torch's current stream there
        with torch.cuda.device(dev):
            field = torch.empty(m["C"] * int(p_i[6]), dtype=torch.float64, device=dev)
            torch.cuda.current_stream(dev).synchronize()
            self.read_device(iid, field)
            mom = ob._moments(m["theory"], field, None, p_i, p_f)
            B = mom[0]
            com = np.zeros(3) if abs(B) < 1.0e-30 else mom[1:4] / B
            rms = 0.0
            if abs(B) >= 1.0e-30:
                num = mom[8] - 2.0 * float(np.dot(com, mom[5:8])) + float(np.dot(com, com)) * mom[4]
                rms = math.sqrt(max(num / B, 0.0))
            out = {"center_of_mass": com, "rms_radius": rms}
            if m["theory"] == 0:
                _, d = ob._nuclear_diag(0, field, None, p_i, p_f, moments=mom)
                E = ob._total("sky_total_energy", 0, field, None, None, None, p_i, p_f)
                out.update(U=ob._sym(d[0:6]), V=ob._sym(d[6:12]), W=d[12:21].reshape(3, 3).copy(),
                           quadrupole=ob._sym(d[21:27]), D_term=-(2.0 / 5.0) * E * float(d[27]))
        return out

    def time_stages(self, nsteps: int) -> dict:
        """Advance nsteps un-captured steps timing each launch kind with CUDA events (ms per step)."""
        out = (ctypes.c_double * 6)()
        self._call("sky_engine_time_stages", int(nsteps), out)
        keys = ("stage1", "stage2", "stage3", "stage4", "control", "advance")
        return dict(zip(keys, list(out)))

    @property
    def launches_per_step(self) -> int:
        return int(self._lib.sky_engine_launches_per_step(self._h))

    def __len__(self):
        return int(self._lib.sky_engine_count(self._h))

    @property
    def bytes(self) -> int:
        return int(self._lib.sky_engine_bytes(self._h))


def instance_bytes(C: int, N: int, precision: str = "fp32") -> int:
    """Device bytes one instance occupies (7 state / slope arrays + small per-tile scratch)."""
    es = 4 if precision == "fp32" else 8
    return 7 * es * C * N + 8192 * 48 + N // 4
