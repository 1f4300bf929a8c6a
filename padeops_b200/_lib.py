"""ctypes binding of libpado.so (the C ABI declared in include/pado.h).

The library is required: importing this module without a built
``_lib/libpado.so`` raises, there is no fallback implementation.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_lib", "libpado.so")

CD06, CD10, CF90 = 0, 1, 2
FILTER, D1, D2 = 0, 1, 2

OK = 0
E_BC = 324
E_NULL, E_ALIAS, E_UNSUPPORTED, E_ARG, E_CUDA, E_SIZE, E_TIMEOUT, E_NOMEM, E_STATE = -1, -2, -3, -4, -5, -6, -7, -8, -9
STATIC_BATCH_MAX_ITEMS = 256  # PADO_STATIC_BATCH_MAX_ITEMS


class PadoError(RuntimeError):
    """A non-zero status returned by the C ABI."""

    def __init__(self, status: int, what: str = ""):
        self.status = status
        msg = lib().pado_strerror(status).decode() if _lib is not None else str(status)
        super().__init__(f"{what}: status {status} ({msg})" if what else f"status {status} ({msg})")


class BatchItem(ctypes.Structure):
    _fields_ = [("op", ctypes.c_void_p), ("kind", ctypes.c_int), ("axis", ctypes.c_int), ("bc1", ctypes.c_int),
                ("bcn", ctypes.c_int), ("n1", ctypes.c_long), ("n2", ctypes.c_long), ("n3", ctypes.c_long),
                ("f", ctypes.c_void_p), ("df", ctypes.c_void_p)]


class HostTerm(ctypes.Structure):
    _fields_ = [("op", ctypes.c_void_p), ("kind", ctypes.c_int), ("axis", ctypes.c_int), ("bc1", ctypes.c_int),
                ("bcn", ctypes.c_int), ("alpha", ctypes.c_double), ("beta", ctypes.c_double), ("out", ctypes.c_int)]


_lib = None

# name -> (restype, argtypes)
_P, _I, _L, _D = ctypes.c_void_p, ctypes.c_int, ctypes.c_long, ctypes.c_double
_APPLY = [_P, _P, _P, _L, _L, _I, _I, _P]
SIGNATURES = {
    "pado_create": (_I, [ctypes.POINTER(_P), _I, _I, _D, _I, _I, _I]),
    "pado_cd06_init": (_I, [ctypes.POINTER(_P), _I, _D, _I, _I, _I]),
    "pado_cd10_init": (_I, [ctypes.POINTER(_P), _I, _D, _I, _I, _I]),
    "pado_cf90_init": (_I, [ctypes.POINTER(_P), _I, _I]),
    "pado_destroy": (None, [_P]),
    "pado_get_size": (_I, [_P]),
    "pado_dd1": (_I, _APPLY), "pado_dd2": (_I, _APPLY), "pado_dd3": (_I, _APPLY),
    "pado_d2d1": (_I, _APPLY), "pado_d2d2": (_I, _APPLY), "pado_d2d3": (_I, _APPLY),
    "pado_filter1": (_I, _APPLY), "pado_filter2": (_I, _APPLY), "pado_filter3": (_I, _APPLY),
    "pado_apply": (_I, [_P, _I, _I, _P, _P, _L, _L, _I, _I, _P]),
    "pado_apply_adjoint": (_I, [_P, _I, _I, _P, _P, _L, _L, _I, _I, _P]),
    "pado_apply_scaled": (_I, [_P, _I, _I, _P, _P, _L, _L, _I, _I, _D, _D, _P]),
    "pado_apply_host": (_I, [_P, _I, _I, _P, _P, _L, _L, _I, _I, _P]),
    "pado_apply_host_terms": (_I, [_P, _L, _L, _L, ctypes.POINTER(HostTerm), _I, ctypes.POINTER(_P), _I, _P]),
    "pado_set_tiling": (_I, [_P, _I, _I]),
    "pado_set_kernel_variant": (_I, [_P, _I]),
    "pado_device_status": (_I, [_P, _I]),
    "pado_set_stream_tiling": (_I, [_P, _I, _I]),
    "pado_launch_plan": (_I, [_P, _I, _I, _P, _P, _L, _L, _I, _I, ctypes.POINTER(_I)]),
    "pado_get_tiling": (_I, [_P, ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "pado_batch_create": (_I, [ctypes.POINTER(_P), ctypes.POINTER(BatchItem), _I]),
    "pado_batch_run": (_I, [_P, _P]),
    "pado_batch_run_loop": (_I, [_P, _P]),
    "pado_batch_run_graph": (_I, [_P, _P]),
    "pado_batch_set_config": (_I, [_P, _I, _I]),
    "pado_batch_info": (_I, [_P, ctypes.POINTER(ctypes.c_longlong), ctypes.POINTER(_I), ctypes.POINTER(_I),
                             ctypes.POINTER(ctypes.c_longlong)]),
    "pado_batch_status": (_I, [_P]),
    "pado_batch_destroy": (None, [_P]),
    "pado_batch_run_static": (_I, [_P, _I, _P]),
    "pado_batch_set_graph_branches": (_I, [_P, _I]),
    "pado_filter3_complex": (_I, [_P, _P, _P, _L, _L, _I, _I, _P]),
    "pado_cd06stagg_init_periodic": (_I, [ctypes.POINTER(_P), _I, _D]),
    "pado_cd06stagg_init_nonperiodic": (_I, [ctypes.POINTER(_P), _I, _D, _I, _I, _I, _I]),
    "pado_cd06stagg_sizes": (_I, [_P, _I, ctypes.POINTER(_I), ctypes.POINTER(_I)]),
    "pado_cd06stagg_apply": (_I, [_P, _I, _P, _P, _L, _L, _P]),
    "pado_cd06stagg_destroy": (None, [_P]),
    "pado_strerror": (ctypes.c_char_p, [_I]),
    "pado_launch_count": (ctypes.c_longlong, []),
    "pado_version": (ctypes.c_char_p, []),
}


def lib() -> ctypes.CDLL:
    """The loaded library (loaded on first use; raises if it was never built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"padeops_b200 CUDA library not built: {LIB_PATH} is missing "
                          "(run `python -m padeops_b200.build`)")
    handle = ctypes.CDLL(LIB_PATH, mode=ctypes.RTLD_GLOBAL)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(handle, name)
        fn.restype = res
        fn.argtypes = args
    _lib = handle
    return _lib


def check(status: int, what: str = "") -> None:
    if status != OK:
        raise PadoError(status, what)
