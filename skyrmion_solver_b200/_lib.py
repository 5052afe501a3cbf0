"""ctypes binding of ``libskyrmion_b200.so`` (the C ABI in ``include/skyrmion_b200.h``).

There is no fallback: if the library is missing or fails to load, importing a
compute path raises ``SkyLibraryError``.  Device buffers may be torch CUDA
tensors or any object exposing ``__cuda_array_interface__`` (Numba device
arrays included); they are passed to the library as raw device pointers.
"""
from __future__ import annotations

import ctypes
import os
import re

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libskyrmion_b200.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "skyrmion_b200.h")

SKY_OK = 0
STATUS_NAMES = {0: "SKY_OK", 1: "SKY_ERR_INVALID", 2: "SKY_ERR_CUDA", 3: "SKY_ERR_NONFINITE",
                4: "SKY_ERR_TIMEOUT", 5: "SKY_ERR_NOMEM"}

THEORY_IDS = {"nuclear": 0, "omega": 1, "coulomb": 2, "rho": 3, "berger": 4, "lightly_bound": 5}


class SkyLibraryError(ImportError):
    pass


class SkyError(RuntimeError):
    """A non-zero sky_status from the library."""

    def __init__(self, status, fn, detail):
        self.status = status
        super().__init__(f"{fn} failed with {STATUS_NAMES.get(status, status)}: {detail}")


class SkyInvalidArgument(SkyError, ValueError):
    pass


_P = ctypes.c_void_p
_I32P = ctypes.POINTER(ctypes.c_int32)
_F64P = ctypes.POINTER(ctypes.c_double)
_F32P = ctypes.POINTER(ctypes.c_float)
_I = ctypes.c_int
_I32 = ctypes.c_int32
_I64 = ctypes.c_int64
_D = ctypes.c_double

# argument signatures of every exported entry point
SIGNATURES = {
    "sky_version": ([], ctypes.c_char_p),
    "sky_last_error": ([], ctypes.c_char_p),
    "sky_set_option": ([_I, _I], _I),
    "sky_get_option": ([_I], _I),
    "sky_theory_components": ([_I], _I),
    "sky_reduce_scratch_size": ([_I64], _I64),
    "sky_gradient_step": ([_I, _I32P, _I32, _F64P, _I32, _P, _P, _P, _P], _I),
    "sky_rk4_stage": ([_I32P, _I32, _F64P, _I32, _P, _P, _P, _P, _P, _P, _D, _P], _I),
    "sky_rk4_finalize": ([_I, _I32P, _I32, _F64P, _I32] + [_P] * 10 + [_P], _I),
    "sky_energy_density": ([_I, _I32P, _I32, _F64P, _I32, _P, _P, _P], _I),
    "sky_baryon_density": ([_I, _I32P, _I32, _F64P, _I32, _P, _P, _P], _I),
    "sky_potential_density": ([_I32P, _I32, _P, _P, _P], _I),
    "sky_rho_meson_density": ([_I32P, _I32, _P, _P, _P], _I),
    "sky_set_field_zero": ([_I32P, _I32, _P, _P], _I),
    "sky_create_grid": ([_I32P, _I32, _F64P, _I32, _P, _P], _I),
    "sky_sum": ([_P, _I64, _P, _I64, _F64P, _P, _P], _I),
    "sky_max": ([_P, _I64, _P, _I64, _F64P, _P, _P], _I),
    "sky_min": ([_P, _I64, _P, _I64, _F64P, _P, _P], _I),
    "sky_arresting_criteria": ([_I32P, _I32, _P, _P, _P, _P, _I64, _F64P, _P], _I),
    "sky_total_energy": ([_I, _I32P, _I32, _F64P, _I32, _P, _P, _I64, _F64P, _P], _I),
    "sky_total_baryon": ([_I, _I32P, _I32, _F64P, _I32, _P, _P, _I64, _F64P, _P], _I),
    "sky_arrested_newton_step": ([_I, _I32P, _I32, _F64P, _I32] + [_P] * 12 + [_P, _I64, _D, _F64P, _F64P, _P],
                                 _I),
    "sky_arrested_newton_step_noalloc": ([_I, _I32P, _I32, _F64P, _I32, _P, _P, _P, _D, _F64P, _F64P, _P], _I),
    "sky_baryon_moments": ([_I, _I32P, _I32, _F64P, _I32, _P, _P, _I64, _F64P, _P], _I),
    "sky_nuclear_diagnostics": ([_I32P, _I32, _F64P, _I32, _P, _F64P, _P, _I64, _F64P, _P], _I),
    "sky_init_field": ([_I32P, _I32, _F64P, _I32, _I32, _I32P, _F64P, _F64P, _D, _I32, _P, _P], _I),
    "sky_init_lumps": ([_I32P, _I32, _F64P, _I32, _I32, _F64P, _I32, _P, _P], _I),
    "sky_volume_scratch_size": ([], _I64),
    "sky_build_rgba_volume": ([_I32P, _I32, _P, _P, _P, _I64, _P, _F64P, _P], _I),
    "sky_render_volume": ([_P, _I32, _I32, _I32, _F32P, _I32, _I32, _I32, _I32, _I32, _P, _P], _I),
    "sky_engine_create": ([_I, ctypes.POINTER(ctypes.c_void_p)], _I),
    "sky_engine_destroy": ([_P], _I),
    "sky_engine_add": ([_P, _I, _I32P, _I32, _F64P, _I32, _I, _P, _P, _I, ctypes.POINTER(_I)], _I),
    "sky_engine_remove": ([_P, _I], _I),
    "sky_engine_set_precision": ([_P, _I, _I], _I),
    "sky_engine_set_active": ([_P, _I, _I], _I),
    "sky_engine_retile": ([_P, _I, _I], _I),
    "sky_engine_set_staging": ([_P, _I, _I, _I], _I),
    "sky_engine_get_staging": ([_P, _I, ctypes.POINTER(_I), ctypes.POINTER(_I)], _I),
    "sky_engine_get_xc": ([_P, _I], _I),
    "sky_engine_set_defect_period": ([_P, _I, _I], _I),
    "sky_engine_audit": ([_P, _I, _F64P], _I),
    "sky_engine_step": ([_P, _I], _I),
    "sky_engine_synchronize": ([_P], _I),
    "sky_engine_stream": ([_P], _P),
    "sky_engine_stats": ([_P, _I, _I64, _F64P], _I),
    "sky_engine_stats_ex": ([_P, _I, _I64, _F64P], _I),
    "sky_engine_stats_all": ([_P, ctypes.POINTER(_I), _F64P, _I, ctypes.POINTER(_I)], _I),
    "sky_engine_read": ([_P, _I, _P, _P, _I], _I),
    "sky_engine_time_stages": ([_P, _I, _F64P], _I),
    "sky_engine_launches_per_step": ([_P], _I),
    "sky_engine_count": ([_P], _I),
    "sky_engine_bytes": ([_P], _I64),
}

_lib = None


def header_symbols(path: str = HEADER):
    """Function names declared in the public header."""
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(sky_[a-z0-9_]+)\s*\(", text)))


def load():
    """Load the shared library (once) and attach the prototypes."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise SkyLibraryError(
            f"{LIB_PATH} is missing: build it with `python -m skyrmion_solver_b200._build` "
            "(there is no CPU fallback)")
    try:
        lib = ctypes.CDLL(LIB_PATH)
    except OSError as e:  # pragma: no cover - depends on the machine
        raise SkyLibraryError(f"cannot load {LIB_PATH}: {e}") from e
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def last_error() -> str:
    return load().sky_last_error().decode()


def check(rc: int, fn: str):
    if rc != SKY_OK:
        detail = last_error()
        if rc == 1:
            raise SkyInvalidArgument(rc, fn, detail)
        raise SkyError(rc, fn, detail)


def call(name: str, *args):
    fn = getattr(load(), name)
    check(fn(*args), name)


# ---------------------------------------------------------------------------
# argument marshalling
# ---------------------------------------------------------------------------

def dptr(buf, dtype="float64"):
    """Raw device pointer of a torch CUDA tensor or a __cuda_array_interface__ object."""
    if buf is None:
        return None
    try:
        import torch
        if isinstance(buf, torch.Tensor):
            if not buf.is_cuda:
                raise ValueError("expected a CUDA tensor, got a CPU tensor")
            if dtype is not None and str(buf.dtype).replace("torch.", "") != dtype:
                raise ValueError(f"expected {dtype} tensor, got {buf.dtype}")
            if not buf.is_contiguous():
                raise ValueError("device buffers must be contiguous")
            return ctypes.c_void_p(buf.data_ptr())
    except ImportError:  # pragma: no cover
        pass
    cai = getattr(buf, "__cuda_array_interface__", None)
    if cai is None:
        raise TypeError(f"{type(buf).__name__} is not a device buffer")
    if dtype is not None and np.dtype(cai["typestr"]) != np.dtype(dtype):
        raise ValueError(f"expected {dtype} device array, got {cai['typestr']}")
    return ctypes.c_void_p(cai["data"][0])


def host_params(p_i, p_f=None):
    """Host int32/float64 copies of the parameter arrays (accepts DeviceParams, numpy or tensors)."""
    def host(a, dt):
        if a is None:
            return None
        h = getattr(a, "host", None)
        if h is not None:
            return np.ascontiguousarray(h, dtype=dt)
        try:
            import torch
            if isinstance(a, torch.Tensor):
                return np.ascontiguousarray(a.detach().cpu().numpy(), dtype=dt)
        except ImportError:  # pragma: no cover
            pass
        if hasattr(a, "copy_to_host"):
            return np.ascontiguousarray(a.copy_to_host(), dtype=dt)
        return np.ascontiguousarray(np.asarray(a), dtype=dt)
    return host(p_i, np.int32), host(p_f, np.float64)


def i32p(a):
    return a.ctypes.data_as(_I32P)


def f64p(a):
    return a.ctypes.data_as(_F64P)


def f32p(a):
    return a.ctypes.data_as(_F32P)


def stream_ptr(stream=None):
    if stream is not None:
        return ctypes.c_void_p(int(getattr(stream, "cuda_stream", stream)))
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
