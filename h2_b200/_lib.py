"""ctypes binding of libh2g.so (the C ABI declared in include/h2g.h).

The library is the product path: if it is missing or cannot be loaded, every call raises
``H2GLibraryError``.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libh2g.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "h2g.h")

H2G_OK, H2G_NOT_CONVERGED, H2G_BREAKDOWN, H2G_NONFINITE = 0, 1, 2, 3
H2G_BAD_ARG, H2G_CUDA_ERROR, H2G_TIMEOUT, H2G_UNSUPPORTED = 4, 5, 6, 7
H2G_FP64, H2G_MIXED, H2G_MIXED_IR = 0, 1, 2
H2G_SMOOTHER_NONE, H2G_SMOOTHER_GS = 0, 1
H2G_ISOTHERMAL, H2G_HEAT_FLUX, H2G_CONVECTION = 0, 1, 2


class H2GLibraryError(RuntimeError):
    """libh2g.so is missing or failed to load (the CUDA path is required)."""


class H2GError(RuntimeError):
    def __init__(self, status: int, msg: str):
        super().__init__(f"h2g status {status}: {msg}")
        self.status = status


class Bc(C.Structure):
    _fields_ = [("type", C.c_int), ("temperature", C.c_double), ("heat_flux", C.c_double),
                ("htc", C.c_double), ("ambient", C.c_double)]


class Result(C.Structure):
    _fields_ = [("isconverged", C.c_int), ("itr", C.c_int), ("outer", C.c_int), ("status", C.c_int),
                ("res0", C.c_double), ("res", C.c_double), ("launches", C.c_longlong)]


_dp = C.POINTER(C.c_double)
_vp = C.c_void_p
_ip = C.POINTER(C.c_int)

# name -> (restype, argtypes)
_SIGS = {
    "h2g_version": (C.c_char_p, []),
    "h2g_status_string": (C.c_char_p, [C.c_int]),
    "h2g_last_error": (C.c_char_p, []),
    "h2g_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(_vp)]),
    "h2g_destroy": (C.c_int, [_vp]),
    "h2g_set_stream": (C.c_int, [_vp, _vp]),
    "h2g_set_grid": (C.c_int, [_vp, _dp, _dp, C.c_double, C.c_double, C.c_double, _dp, C.c_int]),
    "h2g_set_fields": (C.c_int, [_vp, _dp, _dp, _dp, _dp]),
    "h2g_set_rhs": (C.c_int, [_vp, _dp]),
    "h2g_get_rhs": (C.c_int, [_vp, _dp]),
    "h2g_set_theta": (C.c_int, [_vp, _dp]),
    "h2g_get_theta": (C.c_int, [_vp, _dp]),
    "h2g_theta_snapshot": (C.c_int, [_vp, C.c_int]),
    "h2g_set_mixed_params": (C.c_int, [_vp, C.c_double, C.c_int]),
    "h2g_pbicgstab": (C.c_int, [_vp, C.c_double, C.c_int, C.c_int, C.c_int, _dp, C.POINTER(Result)]),
    "h2g_cg": (C.c_int, [_vp, C.c_double, C.c_int, C.c_int, C.c_int, _dp, C.POINTER(Result)]),
    "h2g_PBiCGSTAB": (C.c_int, [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, C.c_double, C.c_double,
                                C.c_double, _dp, _dp, _dp, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                _dp, C.POINTER(Result)]),
    "h2g_CG": (C.c_int, [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, C.c_double, C.c_double,
                         C.c_double, _dp, _dp, _dp, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                         _dp, C.POINTER(Result)]),
    "h2g_sor": (C.c_int, [_vp, C.c_double, C.c_double, C.c_int, C.c_int, _dp, C.POINTER(Result)]),
    "h2g_SolveSOR": (C.c_int, [C.c_int, C.c_int, C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, C.c_double, C.c_double,
                               C.c_double, C.c_double, _dp, _dp, _dp, C.c_double, C.c_int, C.c_int, C.c_int, _dp,
                               C.POINTER(Result)]),
    "h2g_set_hsrc": (C.c_int, [_vp, _dp]),
    "h2g_calrhs": (C.c_int, [_vp, C.POINTER(Bc), C.c_int]),
    "h2g_transient": (C.c_int, [_vp, C.POINTER(Bc), C.c_int, C.c_int, C.c_double, C.c_int, C.c_int, C.c_int, _dp,
                                C.POINTER(Result)]),
    "h2g_batch_solve": (C.c_int, [C.c_int, C.POINTER(C.c_void_p), C.c_int, C.c_double, C.c_int, C.c_int, C.c_int,
                                  C.POINTER(Result)]),
    "h2g_adjoint": (C.c_int, [_vp, _dp, C.c_double, C.c_double, C.c_int, C.c_int, _dp, _dp, _dp,
                              C.POINTER(Result), C.POINTER(Result)]),
    "h2g_adjoint_transient": (C.c_int, [_vp, C.POINTER(Bc), C.c_int, _dp, C.c_double, C.c_double, C.c_int, C.c_int,
                                        C.c_int, _dp, _dp, _dp, C.POINTER(Result)]),
    "h2g_autotune": (C.c_int, [_vp, _ip, _ip, _ip, _ip]),
    "h2g_set_tuning": (C.c_int, [_vp, C.c_int, C.c_int]),
    "h2g_create_multi": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(_vp)]),
    "h2g_set_rhs_multi": (C.c_int, [_vp, _dp]),
    "h2g_set_theta_multi": (C.c_int, [_vp, _dp]),
    "h2g_get_theta_multi": (C.c_int, [_vp, _dp]),
    "h2g_pbicgstab_multi": (C.c_int, [_vp, C.c_double, C.c_int, C.c_int, C.POINTER(Result)]),
    "h2g_set_sweep": (C.c_int, [_vp, C.c_int, C.c_int, C.c_int]),
    "h2g_get_sweep": (C.c_int, [_vp, _ip, _ip, _ip]),
    "h2g_set_coop": (C.c_int, [_vp, C.c_int]),
    "h2g_get_coop": (C.c_int, [_vp, _ip]),
    "h2g_set_wait_limit": (C.c_int, [_vp, C.c_longlong]),
    "h2g_release_cached": (C.c_int, []),
    "h2g_calcax": (C.c_int, [_vp, _dp, _dp]),
    "h2g_calcrk": (C.c_int, [_vp, _dp, _dp]),
    "h2g_rbsor_pass": (C.c_int, [_vp, _dp, _dp, C.c_int, C.c_double]),
    "h2g_preconditioner": (C.c_int, [_vp, _dp, _dp, C.c_int]),
    "h2g_bench_kernel": (C.c_int, [_vp, C.c_int, C.c_int, _ip]),
    "h2g_calcrk_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_int, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                     C.c_double, C.c_double, C.c_double, _dp, C.c_int, _vp, _dp, _vp]),
    "h2g_model_zgrid": (C.c_int, [C.c_int, _dp, _dp, _dp]),
    "h2g_model_pitch": (C.c_double, [C.c_int]),
    "h2g_model_fill_id": (C.c_int, [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint8)]),
}

_lib = None


def header_functions() -> list[str]:
    """Names of the functions declared in include/h2g.h."""
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(h2g_\w+)\s*\(", text)))


def load(path: str | None = None):
    """Load libh2g.so (built by h2_b200/build.py) and declare its signatures."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise H2GLibraryError(f"{p} not found: build it with `python -m h2_b200.build` (nvcc, sm_100a)")
    try:
        lib = C.CDLL(p)
    except OSError as e:  # pragma: no cover - depends on the machine
        raise H2GLibraryError(f"cannot load {p}: {e}") from e
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def last_error() -> str:
    return load().h2g_last_error().decode()


def check(status: int, allowed=(H2G_OK,)) -> int:
    if status not in allowed:
        raise H2GError(status, last_error())
    return status
