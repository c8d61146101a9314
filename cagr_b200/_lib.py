"""ctypes binding of libcagr_b200.so (the C ABI in include/cagr.h).

The library is required: there is no CPU fallback.  Importing works on a
machine without a GPU (the .so links the CUDA runtime statically and only
touches the device when a function is called), so the CPU test suite can
check that every declared symbol is exported.
"""
from __future__ import annotations

import ctypes
import os
import re

from .build import LIB_PATH, ROOT

HEADER = os.path.join(ROOT, "include", "cagr.h")

# status codes (include/cagr.h)
CAGR_OK = 0
CAGR_ERR_ALLOC = 3    # device allocation failed (include/cagr.h)
# dtypes
CAGR_F32, CAGR_F64 = 0, 1
# operators
OPS = {"A": 0, "AT": 1, "A3": 2, "A21": 3, "A22": 4, "A23": 5, "A2T1": 6, "A2T2": 7,
       "A2T3": 8, "G": 9, "A2_FUSED": 10, "A2T_SUM": 11, "COUNT": 12, "A2T_SUM_SHARED": 13,
       "A2_INSIDE": 14, "A2T_RHS": 15}
# far-field modes
FAR_REFERENCE, FAR_INTERP = 0, 1
# multiply flags
FLAG_CONTINUOUS = 1
FLAG_ACCUMULATE = 2
FLAG_NEGATE = 4
ATTR_DIM = {"A": 3, "AT": 1, "A3": 3, "A21": 3, "A22": 3, "A23": 3, "A2T1": 1, "A2T2": 1,
            "A2T3": 1, "G": 3, "A2_FUSED": 3, "A2T_SUM": 3, "A2T_SUM_SHARED": 1, "A2_INSIDE": 3,
            "A2T_RHS": 3}
OUT_DIM = {"A": 1, "AT": 3, "A3": 1, "A21": 1, "A22": 1, "A23": 1, "A2T1": 3, "A2T2": 3,
           "A2T3": 3, "G": 3, "A2_FUSED": 3, "A2T_SUM": 3, "A2T_SUM_SHARED": 3, "COUNT": 1,
           "A2_INSIDE": 4, "A2T_RHS": 3}

_p = ctypes.c_void_p
_i64 = ctypes.c_int64
_i32 = ctypes.c_int
_pp = ctypes.POINTER(ctypes.c_void_p)
_pi64 = ctypes.POINTER(ctypes.c_int64)

_SIGNATURES = {
    "cagr_version": (_i32, []),
    "cagr_status_string": (ctypes.c_char_p, [_i32]),
    "cagr_last_error": (ctypes.c_char_p, []),
    "cagr_tree_build": (_i32, [_p, _i64, _i32, _i32, _i32, _p, _pp]),
    "cagr_tree_destroy": (_i32, [_p]),
    "cagr_tree_info": (_i32, [_p, _pi64, _pi64, _pi64, _pi64, _pi64]),
    "cagr_tree_export": (_i32, [_p] * 9),
    "cagr_tree_morton_order": (_i32, [_p, _p, _p]),
    "cagr_scatter": (_i32, [_p, _i32, _p, _i32, _p, _p]),
    "cagr_scatter3": (_i32, [_p, _p, _p]),
    "cagr_scatter_import": (_i32, [_p, _i32, _p, _p, _p, _i32, _p]),
    "cagr_scatter_export": (_i32, [_p, _i32, _p, _p, _p, _p]),
    "cagr_multiply": (_i32, [_p, _i32, _p, _p, _i64, _p, ctypes.c_double, _i32, _p, _i64, _p]),
    "cagr_forward": (_i32, [_p, _i32, _p, _p, ctypes.c_double, _i32, _p, _p]),
    "cagr_probe_fp32_peak": (_i32, [_i64, ctypes.POINTER(ctypes.c_double), _p]),
    "cagr_probe_rsqrt64": (_i32, [_p, _p, _i64, _p]),
    "cagr_field_grid": (_i32, [_p, _i32, _i32, _i32, _i32, ctypes.POINTER(ctypes.c_double),
                               ctypes.c_double, _p, ctypes.c_double, _i32, _p, _p]),
    "cagr_marching_cubes": (_i32, [_p, _i32, _i32, _i32, ctypes.POINTER(ctypes.c_double),
                                   ctypes.c_double, ctypes.c_double, _p, _i64, _p, _i64, _pi64,
                                   _pi64, _p]),
    "cagr_marching_cubes_table": (_i32, [_p, _i32, _i32, _i32, ctypes.POINTER(ctypes.c_double),
                                         ctypes.c_double, ctypes.c_double, _p, _p, _i64, _p,
                                         _i64, _pi64, _pi64, _p]),
    "cagr_mc_table": (_i32, [_p, _p]),
    "cagr_scatter_noalloc": (_i32, [_p] * 6 + [_i64, _i32, _p, _p, _p, _i32, _p, _p, _p, _p]),
    "cagr_pool_trim": (_i32, [_i64]),
    "cagr_adjoint": (_i32, [_p, _i32, _p, ctypes.c_double, _i32, _p, _p, _p]),
    "cagr_pool_reserved": (_i32, [_pi64, _pi64]),
    "cagr_debug_fail_allocations_after": (_i32, [_i64]),
    "cagr_multiply_rhs_window": (_i32, [_p, _p, ctypes.c_double, _p, _i32, _p, _p]),
    "cagr_b_window_table": (_i32, [_p, _p, _p, _i32, _p, _p]),
    "cagr_tree_set_far_field": (_i32, [_p, _i32, _i32, ctypes.c_double, _i32, _p]),
    "cagr_tree_far_field": (_i32, [_p, ctypes.POINTER(_i32), ctypes.POINTER(_i32),
                                   ctypes.POINTER(ctypes.c_double), ctypes.POINTER(_i32), _pi64]),
    "cagr_tree_query_groups": (_i32, [_p, _p, _p]),
    "cagr_debug_interp_wait_limit": (_i32, [_p, _i64]),
}

_lib = None


class CagrError(RuntimeError):
    """A cagr_* call returned a non-zero status (`code`: the CAGR_ERR_* value)."""

    def __init__(self, message: str, code: int = 0):
        super().__init__(message)
        self.code = code


def header_symbols() -> list[str]:
    """Names of every function declared in include/cagr.h."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\**\s+\**(cagr_\w+)\s*\(", text, re.M)))


def lib() -> ctypes.CDLL:
    """The loaded library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        path = os.environ.get("CAGR_B200_LIB", LIB_PATH)  # an alternative build of the same ABI
        if not os.path.exists(path):
            raise RuntimeError(
                f"{path} is missing: build it with `python -m cagr_b200.build` "
                "(the treecode has no CPU fallback)")
        L = ctypes.CDLL(path)
        for name, (res, args) in _SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int, what: str = "") -> None:
    if rc != CAGR_OK:
        L = lib()
        msg = L.cagr_last_error().decode(errors="replace")
        kind = L.cagr_status_string(rc).decode()
        raise CagrError(f"{what}: {kind} ({rc}): {msg}", rc)
