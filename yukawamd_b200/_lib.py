"""Loader of the engine's C-ABI library (libyukawa_b200.so).

The library is built in-tree by yukawamd_b200.build (nvcc, sm_100a).  There is
no fallback: if the library is missing or does not load, every entry point of
this package raises.
"""
import ctypes as C
import os

from . import abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libyukawa_b200.so")

_lib = None

_dp = C.POINTER(C.c_double)
_P = C.POINTER(abi.YkParams)
_S = C.POINTER(abi.YkScalars)
_ctx = C.c_void_p

# name -> (restype, argtypes); every entry point declared in include/*.h
SIGNATURES = {
    "yk_params_default": (C.c_int, [_P]),
    "yk_create": (C.c_int, [_P, C.c_int, _dp, _dp, _dp, _dp, C.POINTER(_ctx)]),
    "yk_destroy": (C.c_int, [_ctx]),
    "yk_last_error": (C.c_char_p, [_ctx]),
    "yk_accel": (C.c_int, [_ctx, C.c_int, _dp, _S]),
    "yk_newton": (C.c_int, [_ctx, C.c_int, _S]),
    "yk_run": (C.c_int, [_ctx, C.c_int, C.c_int, _S]),
    "yk_get_state": (C.c_int, [_ctx, _dp, _dp, _dp, _dp]),
    "yk_set_state": (C.c_int, [_ctx, _dp, _dp, _dp, _dp]),
    "yk_set_box": (C.c_int, [_ctx, _dp]),
    "yk_snapshot_begin": (C.c_int, [_ctx, _dp, _dp, _dp]),
    "yk_snapshot_wait": (C.c_int, [_ctx]),
    "yk_ttot": (C.c_int, [_ctx, _dp]),
    "yk_vtot": (C.c_int, [_ctx, _dp, _dp]),
    "yk_gofr_counts": (C.c_int, [_ctx, C.c_int, _dp]),
    "yk_tnorm": (C.c_int, [_ctx]),
    "yk_cancel_vcom": (C.c_int, [_ctx]),
    "yk_strain": (C.c_int, [_ctx, _dp, _dp, _dp]),
    "yk_batch_create": (C.c_int, [C.c_int, _P, C.POINTER(C.c_int), C.POINTER(_dp), C.POINTER(_dp),
                                  C.POINTER(_dp), C.POINTER(_dp), C.c_int, C.POINTER(_ctx)]),
    "yk_batch_destroy": (C.c_int, [_ctx]),
    "yk_batch_get_tuning": (C.c_int, [_ctx, C.POINTER(abi.YkTuning)]),
    "yk_batch_set_tuning": (C.c_int, [_ctx, C.POINTER(abi.YkTuning)]),
    "yk_batch_last_error": (C.c_char_p, [_ctx]),
    "yk_batch_accel": (C.c_int, [_ctx, C.c_int, _S]),
    "yk_batch_run": (C.c_int, [_ctx, C.c_int, C.c_int, _S, C.POINTER(C.c_double)]),
    "yk_batch_get_state": (C.c_int, [_ctx, C.c_int, _dp, _dp, _dp, _dp]),
    "yk_batch_set_state": (C.c_int, [_ctx, C.c_int, _dp, _dp, _dp, _dp]),
    "yk_batch_create_slots": (C.c_int, [_P, C.c_int, C.c_longlong, C.c_longlong, C.c_int, C.POINTER(_ctx)]),
    "yk_batch_admit": (C.c_int, [_ctx, _P, C.c_int, _dp, _dp, _dp, _dp, C.c_longlong, C.POINTER(C.c_int), _S]),
    "yk_batch_retire": (C.c_int, [_ctx, C.c_int, _dp, _dp, _dp, _dp]),
    "yk_batch_steps_left": (C.c_int, [_ctx, C.POINTER(C.c_int)]),
    "yk_get_tuning": (C.c_int, [_ctx, C.POINTER(abi.YkTuning)]),
    "yk_set_tuning": (C.c_int, [_ctx, C.POINTER(abi.YkTuning)]),
    "yk_perf_enable": (C.c_int, [_ctx, C.c_int, C.c_size_t]),
    "yk_perf_read": (C.c_int, [_ctx, C.POINTER(abi.YkPerf)]),
    "yk_peak_probe": (C.c_int, [C.c_int, C.c_int, C.POINTER(C.c_double)]),
    "yk_pair_jobs": (C.c_longlong, [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.c_longlong,
                                    C.POINTER(C.c_int)]),
    "yk_pair_jobs2": (C.c_longlong, [C.c_int, C.c_int, C.c_int, C.POINTER(C.c_int), C.c_longlong,
                                     C.POINTER(C.c_int)]),
    "yk_accel_noalloc": (C.c_int, [_P, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int,
                                   C.c_void_p, _S, C.c_void_p]),
    "yk_wait_selftest": (C.c_int, [_ctx, C.c_longlong, C.POINTER(C.c_int)]),
    "yk_host_register": (C.c_int, [C.c_void_p, C.c_size_t]),
    "yk_host_unregister": (C.c_int, [C.c_void_p]),
    "yk_kernel_launch_count": (C.c_ulonglong, []),
    "yk_version": (C.c_char_p, []),
}


class EngineError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("%s: %s" % (abi.STATUS_NAMES.get(code, code), msg))
        self.code = code


def lib():
    """Load (once) and return the ctypes handle; raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError("%s is missing: build it with `python -m yukawamd_b200.build`"
                          % LIB_PATH)
    h = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        f = getattr(h, name)
        f.restype = res
        f.argtypes = args
    _lib = h
    return h


def check(code, ctx=None):
    if code != abi.YK_OK:
        msg = lib().yk_last_error(ctx)
        raise EngineError(code, msg.decode() if msg else "")


def check_batch(code, b=None):
    if code != abi.YK_OK:
        msg = lib().yk_batch_last_error(b)
        raise EngineError(code, msg.decode() if msg else "")
