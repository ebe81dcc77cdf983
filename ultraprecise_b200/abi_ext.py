"""Prototypes of the entry points declared in include/ultraprecise_util.h,
include/ultraprecise_batch.h, ultraprecise_serve.h and
ultraprecise_costmodel.h."""
import ctypes as C

_P = C.c_void_p
_I32 = C.c_int32
_I64 = C.c_int64
_U64 = C.c_uint64

SIGNATURES = {
    "up_util_gen_digits": (_I32, [_P, _I64, _I32, _U64, _I32, _I32, _P]),
    "up_util_gen_range": (_I32, [_P, _I64, _I32, _I64, _I64, _I64, _U64, _P]),
    "up_util_flush_l2": (_I32, [_P, _I64, _P]),
    "up_util_imad_peak": (_I32, [C.POINTER(C.c_double), _P]),
    "up_util_wait_timeout_probe": (_I32, [C.c_uint32, _P, _P, _P]),
    "up_util_compile_only": (_I32, [_P, _I32, _I32, _P, _I32, _I32, _P, _I32]),
    "up_util_compile_expr_only": (_I32, [_P, _I32, _I32, _P, _I32, _P]),
    "up_util_expr_source": (_I64, [_P, _I32, _I32, _P, _I32, _P, C.c_char_p, _I64]),
    # ultraprecise_batch.h
    "up_batch_create": (_I32, [_P, _I32, _P, C.POINTER(_P)]),
    "up_batch_bind": (_I32, [_P, _I32, _P, _I32, _I64, _P, _I32, _P]),
    "up_batch_launch": (_I32, [_P, _P, _P]),
    "up_batch_shape": (_I32, [_P, _I32, C.POINTER(_I32), C.POINTER(_I32), C.POINTER(_I32), C.POINTER(C.c_double)]),
    "up_batch_task_type": (_I32, [_P, _I32, C.POINTER(_I32), C.POINTER(_I32), C.POINTER(_I32), C.POINTER(_I32)]),
    "up_batch_release": (None, [_P]),
    "up_util_compile_batch_only": (_I32, [_P, _I32, _P]),
    "up_batch_task_tpv": (_I32, [_P, _I32, _P]),
    "up_batch_set_task_tpv": (_I32, [_P, _I32, _I32]),
    "up_util_batch_tpv_candidates": (_I32, [_P, _P, _I32]),
    "up_util_auto_tpv": (_I32, [_P, _I32, _I32, _P, _I32, _I32, _P]),
    "up_costmodel_add_member": (_I32, [_P, _P]),
    "up_costmodel_set_guard": (_I32, [_P, C.c_float]),
    # ultraprecise_serve.h
    "up_serve_create": (_I32, [_P, C.POINTER(_P)]),
    "up_serve_clock_ms": (C.c_double, [_P]),
    "up_serve_submit": (_I32, [_P, _P, C.POINTER(_I64)]),
    "up_serve_poll": (_I32, [_P, _I64, C.POINTER(_I32), C.POINTER(C.c_double)]),
    "up_serve_wait": (_I32, [_P, _I64, C.c_double, C.POINTER(_I32)]),
    "up_serve_result": (_I32, [_P, _I64, _I32, C.POINTER(_P), C.POINTER(_I64), C.POINTER(C.c_uint32)]),
    "up_serve_release": (_I32, [_P, _I64]),
    "up_serve_stats_get": (_I32, [_P, _I32, _P]),
    "up_serve_destroy": (None, [_P]),
    # ultraprecise_costmodel.h
    "up_costmodel_create": (_I32, [_U64, C.POINTER(_P)]),
    "up_costmodel_release": (None, [_P]),
    "up_costmodel_expr_features": (_I32, [_P, _I32, _I32, _P, _I32, _I32, _I64, _P, C.POINTER(_I32)]),
    "up_costmodel_train": (_I32, [_P, _P, _P, _I32, _I32, _I32, C.c_float, _U64, C.POINTER(C.c_float)]),
    "up_costmodel_predict": (_I32, [_P, _P, _I32, _P]),
    "up_costmodel_gradients": (_I32, [_P, _P, _P, _I32, _P, C.POINTER(C.c_float)]),
    "up_costmodel_get_params": (_I32, [_P, _P, _P]),
    "up_costmodel_set_params": (_I32, [_P, _P, _P]),
    "up_costmodel_choose_tpv": (_I32, [_P, _P, _I32, _I32, _P, _I32, _I64, C.POINTER(_I32), C.POINTER(C.c_float)]),
    "up_costmodel_set_default": (_I32, [_P]),
}
