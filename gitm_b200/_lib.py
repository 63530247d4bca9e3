"""ctypes binding of libgitmvert.so (the C ABI of include/gitm_vert.h).

The library is the only compute path: loading fails loudly when it is
missing, and nothing here computes a step on the CPU.
"""
from __future__ import annotations

import ctypes as C
import os

from . import abi

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("GITM_VERT_LIB") or os.path.join(_HERE, "libgitmvert.so")
_LIB = None

# Every symbol include/gitm_vert.h declares, with (restype, argtypes).
_P = C.c_void_p
SIGNATURES = {
    "gitm_vert_version": (C.c_char_p, []),
    "gitm_vert_default_params": (None, [C.POINTER(abi.GitmVertParams)]),
    "gitm_vert_create": (C.c_int, [C.POINTER(abi.GitmVertParams), C.c_int, C.POINTER(_P)]),
    "gitm_vert_destroy": (C.c_int, [_P]),
    "gitm_vert_last_error": (C.c_char_p, [_P]),
    "gitm_vert_set_params": (C.c_int, [_P, C.POINTER(abi.GitmVertParams)]),
    "gitm_vert_plan_create": (C.c_int, [_P, C.POINTER(abi.GitmColumnBatch), C.c_int, C.POINTER(_P)]),
    "gitm_vert_plan_destroy": (C.c_int, [_P]),
    "gitm_vert_plan_set_config": (C.c_int, [_P, C.POINTER(abi.GitmLaunchConfig)]),
    "gitm_vert_plan_get_config": (C.c_int, [_P, C.POINTER(abi.GitmLaunchConfig)]),
    "gitm_vert_plan_advance": (C.c_int, [_P, C.c_double, C.c_int, _P]),
    "gitm_vert_plan_autotune": (C.c_int, [_P, C.c_double, C.c_int, C.POINTER(abi.GitmLaunchConfig)]),
    "gitm_vert_plan_status": (C.c_int, [_P, C.POINTER(C.c_uint32), C.POINTER(C.c_int64), C.c_int]),
    "gitm_vert_plan_status_words": (_P, [_P]),
    "gitm_vert_plan_wait": (C.c_int, [_P, _P, C.c_double]),
    "gitm_vert_plan_launch_count": (C.c_int, [_P, C.c_int]),
    "gitm_vert_advance_native": (C.c_int, [_P, C.POINTER(abi.GitmColumnBatch), C.c_int, C.c_double,
                                           C.c_int]),
    "gitm_vert_advance_native_host": (C.c_int, [_P, C.POINTER(abi.GitmColumnBatch), C.c_int,
                                                C.c_double, C.c_int]),
    "gitm_vert_advance_native_noalloc": (C.c_int, [_P, C.POINTER(abi.GitmColumnBatch), C.c_double,
                                                   C.c_int, _P, _P]),
    "gitm_vert_advance_1d": (C.c_int, [_P, C.POINTER(abi.GitmModVerticalBatch), C.c_double, _P]),
    "gitm_vert_plan_adjoint": (C.c_int, [_P, C.POINTER(abi.GitmColumnAdjoint), C.c_double, _P, _P]),
    "gitm_vert_plan_saved_state_doubles": (C.c_int64, [_P]),
    "gitm_vert_plan_advance_saving": (C.c_int, [_P, C.c_double, _P, _P]),
    "gitm_vert_cfl_dt": (C.c_int, [_P, C.POINTER(abi.GitmColumnBatch), C.c_int, C.c_double,
                                   C.c_double, C.c_double, C.POINTER(C.c_double)]),
    "gitm_vert_advance_fortran": (C.c_int, [_P, C.POINTER(abi.GitmFortranState), C.c_int, C.c_int,
                                            C.c_double, C.c_int]),
    # include/gitm_hz.h
    "gitm_hz_advance": (C.c_int, [_P, C.POINTER(abi.GitmHzParams), C.POINTER(abi.GitmHzBlocks), C.c_double, _P]),
    "gitm_hz_status": (C.c_int, [_P, C.POINTER(C.c_uint32), C.POINTER(C.c_int64), C.c_int]),
    "gitm_hz_exchange": (C.c_int, [_P, C.POINTER(abi.GitmHzExchange), _P]),
}


class LibraryMissing(RuntimeError):
    pass


def lib():
    """The loaded library; raises LibraryMissing when it was not built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise LibraryMissing(
                f"{LIB_PATH} is missing: build it with `python -m gitm_b200.build` "
                "(nvcc for sm_100a); there is no CPU fallback")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB
