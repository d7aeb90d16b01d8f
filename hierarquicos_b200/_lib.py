"""ctypes binding of the C ABI declared in include/hierarquicos_bh.h.

The library is the in-tree ``libhierarquicos_bh.so`` (built by
``hierarquicos_b200.build``).  There is no fallback: if the library is missing
or cannot be loaded, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libhierarquicos_bh.so")

BH_OK = 0
BH_ERR_INVALID = 1
BH_ERR_CUDA = 2
BH_ERR_NOMEM = 3
BH_ERR_NONFINITE = 4
BH_ERR_CAPACITY = 5
BH_ERR_DUPLICATES = 6
BH_ERR_INTERNAL = 7
BH_ERR_NOT_BUILT = 8

BH_PREC_FP32 = 0
BH_PREC_FP64 = 1
BH_PREC_REFERENCE = 2
BH_PREC_DEHNEN = 3

# every symbol the header declares (checked by the CPU test suite)
EXPORTED = [
    "bh_params_default", "bh_version", "bh_last_error", "bh_compute_forces",
    "bh_compute_forces_ex", "bh_compute_forces_direct", "bh_direct_targets_device",
    "bh_system_create", "bh_system_destroy", "bh_system_build", "bh_system_walk",
    "bh_system_walk_groups",
    "bh_system_forces", "bh_system_sync", "bh_system_info", "bh_system_get_keys",
    "bh_system_get_nodes", "bh_system_get_groups", "bh_system_get_stats",
    "bh_system_reference_targets", "bh_probe_fma_peak", "bh_probe_bounded_wait", "bh_compute_forces_noalloc",
    "bh_system_build_batch", "bh_system_forces_batch", "bh_system_batch_info",
    "bh_system_capture", "bh_system_replay", "bh_kick_drift", "bh_diagnostics",
    "bh_kick_drift_systems", "bh_generate_ics", "bh_system_reserve", "bh_system_get_key_checks",
]

BH_NOALLOC_MAX_N = 8192


class BHParams(C.Structure):
    """struct bh_params."""

    _fields_ = [
        ("theta", C.c_double), ("G", C.c_double), ("eps", C.c_double),
        ("order", C.c_int), ("out_kind", C.c_int), ("depth", C.c_int), ("precision", C.c_int),
        ("amp", C.c_double), ("group_size", C.c_int), ("leaf_cap", C.c_int),
        ("com_mode", C.c_int), ("strict_keys", C.c_int), ("count_stats", C.c_int),
        ("group_span", C.c_int), ("mac", C.c_int), ("pipeline", C.c_int),
    ]


class BHError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


_lib = None
_lock = threading.Lock()

_vp = C.c_void_p
_i64 = C.c_int64
_d = C.c_double
_i = C.c_int


def lib():
    """Loads the CUDA library; raises if it is missing (no CPU fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `python -m hierarquicos_b200.build`")
        L = C.CDLL(LIB_PATH)
        L.bh_params_default.argtypes = [C.POINTER(BHParams)]
        L.bh_params_default.restype = None
        L.bh_version.restype = C.c_char_p
        L.bh_last_error.argtypes = [C.c_char_p, _i]
        sig = {
            "bh_compute_forces": [_vp, _vp, _vp, _vp, _i64, _d, _d, _d, _i, _i, _vp, _vp],
            "bh_compute_forces_ex": [_vp, _vp, _vp, _vp, _i64, C.POINTER(BHParams), _vp, _vp],
            "bh_compute_forces_direct": [_vp, _vp, _vp, _vp, _i64, _d, _d, _i, _vp, _vp],
            "bh_direct_targets_device": [_vp, _vp, _vp, _vp, _i64, _vp, _i64, _d, _d, _i, _vp, _vp],
            "bh_system_create": [C.POINTER(_vp), _i],
            "bh_system_destroy": [_vp],
            "bh_system_build": [_vp, _vp, _vp, _vp, _vp, _i64, C.POINTER(BHParams), _vp],
            "bh_system_walk": [_vp, C.POINTER(BHParams), _vp, _vp],
            "bh_system_walk_groups": [_vp, C.POINTER(BHParams), _i64, _i64, _vp, _vp],
            "bh_system_forces": [_vp, _vp, _vp, _vp, _vp, _i64, C.POINTER(BHParams), _vp, _vp],
            "bh_system_sync": [_vp, _vp],
            "bh_system_info": [_vp, C.POINTER(_i64), C.POINTER(_i), C.POINTER(_i64),
                               C.POINTER(_i64), _vp, C.POINTER(_d)],
            "bh_system_get_keys": [_vp, _vp, _vp],
            "bh_system_get_nodes": [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
            "bh_system_get_groups": [_vp, _vp],
            "bh_system_get_stats": [_vp, _vp],
            "bh_system_get_key_checks": [_vp, _vp],
            "bh_system_reference_targets": [_vp, C.POINTER(BHParams), _vp, _i64, _vp, _vp, _vp],
            "bh_probe_fma_peak": [_i, _vp],
            "bh_probe_bounded_wait": [_i, C.c_longlong, _vp],
            "bh_compute_forces_noalloc": [_vp, _vp, _vp, _vp, _i64, C.POINTER(BHParams), _vp, _vp],
            "bh_system_build_batch": [_vp, _vp, _vp, _vp, _vp, _vp, _i, C.POINTER(BHParams), _vp],
            "bh_system_forces_batch": [_vp, _vp, _vp, _vp, _vp, _vp, _i, C.POINTER(BHParams), _vp,
                                       _vp],
            "bh_system_batch_info": [_vp, _vp, _vp, _vp],
            "bh_system_capture": [_vp, C.POINTER(BHParams), _vp],
            "bh_system_replay": [_vp, _vp],
            "bh_kick_drift": [_vp] * 8 + [_vp, _i, _i64, _d, _d, _d, _vp],
            "bh_diagnostics": [_vp] * 7 + [_vp, _i, _i64, _d, _d, _vp, _vp, _vp],
            "bh_kick_drift_systems": [_vp] * 8 + [_vp, _i, _i64, _vp, _vp],
            "bh_system_reserve": [_vp, _i64, _i],
            "bh_generate_ics": [_i, _i64, _d, _d, _i, _i, _d, _d, C.c_uint64, _i, _vp, _vp, _vp,
                                _vp, _vp],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = C.c_int
        _lib = L
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(512)
    lib().bh_last_error(buf, 512)
    return buf.value.decode(errors="replace")


def check(rc: int) -> None:
    if rc != BH_OK:
        raise BHError(rc, last_error())


def default_params(**kw) -> BHParams:
    p = BHParams()
    lib().bh_params_default(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise TypeError(f"unknown parameter {k!r}")
        setattr(p, k, v)
    return p
