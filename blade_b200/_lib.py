"""ctypes binding of the blade_b200 C ABI (include/blade_b200.h).

The shared library is built ahead of time (``python -m blade_b200.build``) and
loaded from this package directory.  There is no fallback: if it is missing or
fails to load, every call raises.
"""

from __future__ import annotations

import ctypes as C
import os
import threading

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libblade_b200.so")

# Status codes (Blade::Result).
SUCCESS, ERROR, CUDA_ERROR, ASSERTION_ERROR = 0, 1, 2, 3

# Element types.
I8, I32, F16, F32, F64, CI8, CF16, CF32, CF64 = 1, 2, 3, 4, 5, 6, 7, 8, 9


class BladeError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, what: str, status: int, message: str):
        super().__init__(f"{what}: {message} (status {status})")
        self.status = status


_lock = threading.Lock()
_lib = None

_u64 = C.c_uint64
_vp = C.c_void_p
_int = C.c_int
_dbl = C.c_double
_u64p = C.POINTER(C.c_uint64)

_SIGNATURES = {
    "blade_last_error": (C.c_char_p, []),
    "blade_version": (_int, []),
    "blade_cast": (_int, [_int, _int, _vp, _vp, _u64, _vp]),
    "blade_phasor_from_delays": (_int, [_vp, _vp, _vp, _u64, _u64, _u64, _u64, _dbl, _dbl, _dbl, _u64, _vp]),
    "blade_beamform_f32": (_int, [_vp, _vp, _vp, _u64, _u64, _u64, _u64, _u64, _int, _int, _vp]),
    "blade_beamform_meerkat_f32": (_int, [_vp, _vp, _vp, _u64, _u64, _u64, _u64, _u64, _int, _vp]),
    "blade_channelize_workspace_size": (_u64, [_u64, _u64, _u64, _u64, _u64]),
    "blade_channelize": (_int, [_vp, _vp, _vp, _u64, _u64, _u64, _u64, _u64, _vp]),
    "blade_spectrometer_workspace_size": (_u64, [_u64, _u64, _u64, _u64, _u64]),
    "blade_spectrometer": (_int, [_int, _vp, _int, _vp, _vp, _u64, _u64, _u64, _u64, _u64, _u64, _u64, _int, _vp]),
    "blade_polarize": (_int, [_int, _vp, _vp, _u64, _vp]),
    "blade_detect": (_int, [_vp, _vp, _u64, _u64, _u64, _u64, _u64, _u64, _vp]),
    "blade_gather": (_int, [_u64, _vp, _vp, _u64p, _u64, _u64, _u64, _vp]),
    "blade_permute": (_int, [_u64, _vp, _vp, _u64p, _u64p, _vp]),
    "blade_duplicate": (_int, [_vp, _vp, _u64, _vp]),
    "blade_beamform_detect_f32": (_int, [_int, _vp, _vp, _vp, _u64, _u64, _u64, _u64, _u64, _u64, _u64, _vp]),
    "blade_beamform_tc_plan_size": (_u64, [_u64, _u64, _u64, _u64]),
    "blade_beamform_tc_prepare": (_int, [_vp, _vp, _u64, _u64, _u64, _u64, _vp]),
    "blade_beamform_detect_tc_supported": (_int, [_u64, _u64, _u64, _u64, _u64, _u64, _u64]),
    "blade_beamform_detect_tc": (_int, [_vp, _vp, _vp, _u64, _u64, _u64, _u64, _u64, _u64, _u64, _vp]),
    "blade_beamform_prepare_detect_tc": (_int, [_vp, _vp, _vp, _vp, _u64, _u64, _u64, _u64, _u64, _u64, _u64, _vp]),
    "blade_beamform_prepare_detect_tc_cf16": (_int, [_vp, _vp, _vp, _vp, _u64, _u64, _u64, _u64, _u64, _u64, _vp]),
    "blade_beamform_detect_tc_cf16": (_int, [_vp, _vp, _vp, _u64, _u64, _u64, _u64, _u64, _u64, _vp]),
    "blade_prechannelize_cf16": (_int, [_vp, _vp, _u64, _u64, _u64, _u64, _u64, _int, _vp]),
    "blade_incoherent_detect_cf16": (_int, [_vp, _vp, _vp, _u64, _u64, _u64, _u64, _u64, _vp]),
    "blade_beamform_detect_adjoint": (_int, [_vp, _vp, _vp, _vp, _u64, _u64, _u64, _u64, _u64, _vp]),
    "blade_beamform_detect_adjoint_f32": (_int, [_vp, _vp, _vp, _vp, _u64, _u64, _u64, _u64, _u64, _vp]),
    "blade_beamform_detect_adjoint_tc": (_int, [_vp, _vp, _vp, _vp, _u64, _u64, _u64, _u64, _u64, _vp]),
    "blade_device_status": (_int, [C.POINTER(C.c_uint32)]),
    "blade_wait_selftest": (_int, [_u64, _vp]),
    "blade_beamform_detect_tc_noalloc": (_int, [_vp, _vp, _vp, _u64, _u64, _u64, _u64, _u64, _u64, _u64, _vp]),
    "blade_beamform_detect_tc_autotune": (_int, [_u64, _u64, _u64, _u64, _u64, _u64, _u64, _vp]),
    "blade_beamform_detect_f32_autotune": (_int, [_int, _u64, _u64, _u64, _u64, _u64, _u64, _u64, _vp]),
    "blade_spectrometer_autotune": (_int, [_int, _int, _u64, _u64, _u64, _u64, _u64, _u64, _u64, _vp]),
    "blade_autotune_query": (_int, [_int, _u64p, C.POINTER(C.c_uint32), C.POINTER(C.c_float), C.POINTER(_int)]),
    "blade_autotune_clear": (_int, []),
    "blade_geometric_delays": (_int, [_vp, _u64, _u64, _vp, _dbl, _dbl, _vp, _u64, _dbl, _dbl, _vp, _vp]),
    "blade_source_direction": (_int, [_dbl, _dbl, _dbl, _dbl, C.POINTER(C.c_double)]),
}


def load():
    """Load the shared library once and declare every exported signature."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m blade_b200.build`")
        lib = C.CDLL(LIB_PATH, mode=C.RTLD_GLOBAL)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        return lib


def exported_symbols():
    return list(_SIGNATURES)


def last_error() -> str:
    msg = load().blade_last_error()
    return msg.decode() if msg else ""


def check(status: int, what: str) -> None:
    if status != SUCCESS:
        raise BladeError(what, status, last_error())


def call(name: str, *args) -> int:
    """Call ``name`` and raise BladeError on a non-zero status."""
    st = getattr(load(), name)(*args)
    check(st, name)
    return st


def u64_array(values):
    arr = (C.c_uint64 * len(values))(*[int(v) for v in values])
    return arr
