"""ctypes view of include/ultraprecise.h and the loader of libultraprecise.so.

The library is built in-tree (``ultraprecise_b200/_lib/libultraprecise.so``)
by ``ultraprecise_b200/build.py``.  Loading fails loudly when it is missing:
there is no CPU fallback for any product entry point.
"""
from __future__ import annotations

import ctypes as C
import os

UP_OK = 0
UP_ERR_INVALID_ARG = 1
UP_ERR_UNSUPPORTED = 2
UP_ERR_CUDA = 3
UP_ERR_COMPILE = 4
UP_ERR_NO_MEMORY = 5
UP_ERR_TIMEOUT = 6
UP_ERR_QUEUE_FULL = 7
UP_ERR_NOT_READY = 8
UP_ERR_NO_DEVICE = 9

UP_ROWERR_OVERFLOW = 1
UP_ROWERR_DIV_BY_ZERO = 2
UP_ROWERR_DOMAIN = 4
UP_ROWERR_TIMEOUT = 8

UP_NODE_COLUMN = 0
UP_NODE_CONST = 1
UP_NODE_INT = 2
UP_NODE_ADD = 3
UP_NODE_SUB = 4
UP_NODE_MUL = 5
UP_NODE_DIV = 6
UP_NODE_MOD = 7
UP_NODE_LT = 10
UP_NODE_LE = 11
UP_NODE_GT = 12
UP_NODE_GE = 13
UP_NODE_EQ = 14
UP_NODE_NE = 15
UP_NODE_AND = 16
UP_NODE_OR = 17
UP_NODE_RESCALE = 20
UP_KEY_TABLE_ENTRIES = 131088
UP_KEY_TABLE_COUNT = 131072
COMPARE_KINDS = (UP_NODE_LT, UP_NODE_LE, UP_NODE_GT, UP_NODE_GE, UP_NODE_EQ, UP_NODE_NE, UP_NODE_AND, UP_NODE_OR)

UP_CONST_MAX_LIMBS = 128

UP_AGG_COUNT = 0
UP_AGG_SUM = 1
UP_AGG_AVG = 2
UP_AGG_DECIMAL_BYTES = 133


class UpExprNode(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("left", C.c_int32),
        ("right", C.c_int32),
        ("column", C.c_int32),
        ("precision", C.c_int32),
        ("scale", C.c_int32),
        ("reverse", C.c_int32),
        ("const_sign", C.c_int32),
        ("const_nlimbs", C.c_int32),
        ("int_value", C.c_int64),
        ("const_limbs", C.c_uint32 * UP_CONST_MAX_LIMBS),
    ]


class UpColType(C.Structure):
    _fields_ = [("precision", C.c_int32), ("scale", C.c_int32), ("nullable", C.c_int32)]


class UpColumn(C.Structure):
    _fields_ = [
        ("data", C.c_void_p),
        ("blocks", C.c_void_p),
        ("block_prefix", C.c_void_p),
        ("n_blocks", C.c_int32),
        ("indices", C.c_void_p),
        ("precision", C.c_int32),
        ("scale", C.c_int32),
        ("value_bytes", C.c_int32),
        ("nullable", C.c_int32),
    ]


class UpCompileOpts(C.Structure):
    _fields_ = [("threads_per_value", C.c_int32), ("block_threads", C.c_int32), ("flags", C.c_int32)]


class UpQueryAgg(C.Structure):
    _fields_ = [("kind", C.c_int32), ("root", C.c_int32)]


class UpDeviceInfo(C.Structure):
    _fields_ = [
        ("sm_count", C.c_int32),
        ("cc_major", C.c_int32),
        ("cc_minor", C.c_int32),
        ("free_bytes", C.c_int64),
        ("total_bytes", C.c_int64),
        ("name", C.c_char * 128),
    ]


HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libultraprecise.so")

# name -> (restype, argtypes); every symbol declared in include/ultraprecise.h
_P = C.c_void_p
_I32 = C.c_int32
_I64 = C.c_int64
_PI32 = C.POINTER(C.c_int32)
SIGNATURES = {
    "up_status_string": (C.c_char_p, [_I32]),
    "up_last_error_message": (C.c_char_p, []),
    "up_abi_version": (_I32, []),
    "up_compact_bytes": (_I32, [_I32]),
    "up_precision_words": (_I32, [_I32]),
    "up_max_precision": (_I32, []),
    "up_expr_derive_types": (_I32, [_P, _I32, _I32, _P, _I32]),
    "up_expr_align_optimize": (_I32, [_P, _I32, _I32, _P, _I32, _P, _I32, _PI32, _PI32]),
    "up_module_compile": (_I32, [_P, _I32, _I32, _P, _I32, _P, C.POINTER(_P)]),
    "up_module_result_type": (_I32, [_P, _PI32, _PI32, _PI32]),
    "up_module_source": (_I64, [_P, C.c_char_p, _I64]),
    "up_expr_launch": (_I32, [_P, _P, _I32, _I64, _P, _P, _P]),
    "up_group_table_from_keys": (_I32, [_P, _P, _I32, _I64, _P, _PI32, _P, _P]),
    "up_query_launch_keys": (_I32, [_P, _P, _I32, _I64, _P, _P, _I32, _P, _I32, _P, _P, _P]),
    "up_group_table_from_keys_async": (_I32, [_P, _P, _I32, _I64, _P, _P, _P]),
    "up_query_launch_keys_async": (_I32, [_P, _P, _I32, _I64, _P, _P, _I32, _P, _I32, _P, _P, _P]),
    "up_filter_flags": (_I32, [_P, _I64, _P, _P, _P]),
    "up_parse_decimal": (_I32, [_P, _P, _I64, _I32, _I32, _P, _P, _P]),
    "up_format_width": (_I32, [_I32, _I32]),
    "up_format_decimal": (_I32, [_P, _I64, _I32, _I32, _I32, _P, _I32, _P, _P]),
    "up_expr_launch_host": (_I32, [_P, _P, _I32, _I64, _P, C.POINTER(C.c_uint32), _I64]),
    "up_module_threads_per_value": (_I32, [_P]),
    "up_expr_launch_many": (_I32, [_P, _P, _I32, _P, _I32, _P, _P, _P]),
    "up_module_release": (None, [_P]),
    "up_module_cache_size": (_I32, [_I32]),
    "up_group_agg": (_I32, [_P, _P, _I32, _P, _I32, _I64, _P, _P, _P]),
    "up_aggregate_column_data": (_I32, [_P, _I32, _P, _P, _I32, _I64, _P, _P, _P]),
    "up_division_int64": (_I32, [_P, _P, _I32, _P, _P]),
    "up_group_ids_from_keys": (_I32, [_P, _P, _I32, _I64, _P, _PI32, _P, _P]),
    "up_query_compile": (_I32, [_P, _I32, _P, _I32, _P, _I32, _P, C.POINTER(_P)]),
    "up_query_launch": (_I32, [_P, _P, _I32, _I64, _P, _I32, _P, _P, _P]),
    "up_query_launch_noalloc": (_I32, [_P, _P, _I32, _I64, _P, _I32, _P, _P, _P]),
    "up_device_query": (_I32, [_I32, _P]),
}

_lib = None


class UpError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str):
        super().__init__(f"{where}: status {status} ({status_name(status)}): {detail}")
        self.status = status


def status_name(s: int) -> str:
    names = {0: "OK", 1: "INVALID_ARG", 2: "UNSUPPORTED", 3: "CUDA", 4: "COMPILE", 5: "NO_MEMORY",
             6: "TIMEOUT", 7: "QUEUE_FULL", 8: "NOT_READY", 9: "NO_DEVICE"}
    return names.get(s, "UNKNOWN")


def load(path: str | None = None) -> C.CDLL:
    """Load libultraprecise.so (once).  Raises if it was not built."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"libultraprecise.so not found at {p}: build it with "
            "`python -m ultraprecise_b200.build` (no CPU fallback exists)")
    lib = C.CDLL(p, mode=C.RTLD_GLOBAL)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _declare_extra(lib)
    if path is None:
        _lib = lib
    return lib


def _declare_extra(lib):
    """Prototypes of entry points declared in the other include/*.h headers."""
    from . import abi_ext
    for name, (res, args) in abi_ext.SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args


def check(status: int, where: str) -> None:
    if status != UP_OK:
        lib = load()
        msg = lib.up_last_error_message()
        raise UpError(status, where, msg.decode() if msg else "")
