"""ctypes binding of lib213transpose_b200.so (the C ABI in include/t213.h).

Loading fails loudly when the library has not been built: there is no CPU
fallback anywhere in the package.
"""
from __future__ import annotations

import ctypes
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SO_PATH = os.path.join(HERE, "lib213transpose_b200.so")
HEADER = os.path.join(ROOT, "include", "t213.h")

# status codes (include/t213.h)
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_UNSUPPORTED = 2
ERR_CUDA = 3
ERR_OUT_OF_MEMORY = 4
ERR_TIMEOUT = 5
ERR_BUDGET = 6
ERR_NOT_READY = 7

# plan families
PLAN_AUTO, PLAN_C2R, PLAN_R2C, PLAN_SKINNY, PLAN_BLOCKS, PLAN_BANDS, PLAN_BANDS_T, PLAN_IDENTITY, PLAN_SLICE = range(9)
PLAN_NAMES = {"auto": 0, "c2r": 1, "r2c": 2, "skinny": 3, "blocks": 4, "bands": 5, "bands_t": 6, "identity": 7,
              "slice": 8}


class T213Error(RuntimeError):
    """A non-zero t213_status from the C ABI."""

    def __init__(self, status: int, message: str):
        self.status = status
        super().__init__(f"t213 status {status}: {message}")


class TensorDesc(ctypes.Structure):
    _fields_ = [("data", ctypes.c_void_p), ("d1", ctypes.c_int64), ("d2", ctypes.c_int64), ("d3", ctypes.c_int64),
                ("elem_bytes", ctypes.c_int32), ("plan_kind", ctypes.c_int32)]


class Request(ctypes.Structure):
    _fields_ = [("d1", ctypes.c_int64), ("d2", ctypes.c_int64), ("d3", ctypes.c_int64), ("elem_bytes", ctypes.c_int32),
                ("plan_kind", ctypes.c_int32), ("arrival_s", ctypes.c_double), ("seed", ctypes.c_uint64)]


class ServeStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_int64), ("rejected", ctypes.c_int64), ("bytes_done", ctypes.c_int64),
                ("p50_ms", ctypes.c_double), ("p99_ms", ctypes.c_double), ("mean_ms", ctypes.c_double),
                ("max_ms", ctypes.c_double), ("wall_s", ctypes.c_double), ("peak_resident_bytes", ctypes.c_int64),
                ("max_inflight", ctypes.c_int64), ("cold", ctypes.c_int64), ("p50_cold_ms", ctypes.c_double),
                ("p99_cold_ms", ctypes.c_double), ("p50_warm_ms", ctypes.c_double), ("p99_warm_ms", ctypes.c_double),
                ("group_launches", ctypes.c_int64), ("grouped_requests", ctypes.c_int64)]


_lib = None

_i64, _i32, _vp, _sz = ctypes.c_int64, ctypes.c_int32, ctypes.c_void_p, ctypes.c_size_t
_pi64 = ctypes.POINTER(ctypes.c_int64)
_SIGS = {
    "t213_status_string": ([ctypes.c_int], ctypes.c_char_p),
    "t213_last_error": ([], ctypes.c_char_p),
    "t213_version": ([], ctypes.c_char_p),
    "t213_transpose": ([_vp, _i64, _i64, _i64, _i32, _vp], ctypes.c_int),
    "t213_transpose_with_plan": ([_vp, _i64, _i64, _i64, _i32, _i32, _i64, _vp], ctypes.c_int),
    "t213_c2r_transpose": ([_vp, _i64, _i64, _i64, _i32, _vp], ctypes.c_int),
    "t213_r2c_transpose": ([_vp, _i64, _i64, _i64, _i32, _vp], ctypes.c_int),
    "t213_skinny_c2r_transpose": ([_vp, _i64, _i64, _i64, _i32, _vp], ctypes.c_int),
    "t213_skinny_r2c_transpose": ([_vp, _i64, _i64, _i64, _i32, _vp], ctypes.c_int),
    "t213_rotate": ([_i32, _pi64, _i32, _vp, _i64, _i64, _i64, _i32, _vp], ctypes.c_int),
    "t213_row_shuffle": ([_i32, _pi64, _i32, _vp, _i64, _i64, _i64, _i32, _vp], ctypes.c_int),
    "t213_row_shuffle_noalloc": ([_i32, _pi64, _i32, _vp, _i64, _i64, _i64, _i32, _vp], ctypes.c_int),
    "t213_col_shuffle": ([_i32, _pi64, _i32, _vp, _i64, _i64, _i64, _i32, _vp], ctypes.c_int),
    "t213_scatter_permute": ([_i32, _pi64, _i32, _vp, _i64, _i64, _i64, _i32, _vp], ctypes.c_int),
    "t213_transpose_host": ([_vp, _i64, _i64, _i64, _i32, _vp], ctypes.c_int),
    "t213_permute": ([_vp, _i32, _pi64, ctypes.POINTER(_i32), _i32, _vp], ctypes.c_int),
    "t213_plan_describe": ([_i64, _i64, _i64, _i32, _i32, _i64, ctypes.c_char_p, _sz], ctypes.c_int),
    "t213_plan_launches": ([_i64, _i64, _i64, _i32, _i32, _i64, ctypes.POINTER(_i32)], ctypes.c_int),
    "t213_pass_timing_enable": ([_i32], ctypes.c_int),
    "t213_pass_timing_read": ([ctypes.c_char_p, ctypes.POINTER(ctypes.c_double), _pi64], ctypes.c_int),
    "t213_pass_timing_reset": ([], ctypes.c_int),
    "t213_release_cache": ([], ctypes.c_int),
    "t213_device_status": ([_vp, ctypes.POINTER(_i32)], ctypes.c_int),
    "t213_batch_create": ([ctypes.POINTER(TensorDesc), _i32, ctypes.POINTER(_vp)], ctypes.c_int),
    "t213_batch_execute": ([_vp, _vp], ctypes.c_int),
    "t213_batch_status": ([_vp, _vp], ctypes.c_int),
    "t213_batch_describe": ([_vp, ctypes.c_char_p, _sz], ctypes.c_int),
    "t213_batch_debug_stall": ([_vp, _i64, _i32], ctypes.c_int),
    "t213_batch_destroy": ([_vp], ctypes.c_int),
    "t213_transpose_looped": ([ctypes.POINTER(TensorDesc), _i32, _vp], ctypes.c_int),
    "t213_batch_tune": ([ctypes.POINTER(TensorDesc), _i32, _vp], ctypes.c_int),
    "t213_tune_shape": ([_vp, _i64, _i64, _i64, _i32, _vp, ctypes.POINTER(_i32), _pi64], ctypes.c_int),
    "t213_tuner_load": ([ctypes.c_char_p], ctypes.c_int),
    "t213_tuner_save": ([ctypes.c_char_p], ctypes.c_int),
    "t213_tuner_clear": ([], ctypes.c_int),
    "t213_tuner_lookup": ([_i64, _i64, _i64, _i32, ctypes.POINTER(_i32), _pi64], ctypes.c_int),
    "t213_server_create": ([_i64, _i32, _i32, ctypes.POINTER(_vp)], ctypes.c_int),
    "t213_server_run": ([_vp, ctypes.POINTER(Request), _i32, ctypes.POINTER(ServeStats),
                         ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_double)], ctypes.c_int),
    "t213_server_run_capture": ([_vp, ctypes.POINTER(Request), _i32, ctypes.POINTER(ServeStats),
                                 ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_double),
                                 ctypes.POINTER(_vp)], ctypes.c_int),
    "t213_server_expected_checksum": ([_vp, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_uint64)], ctypes.c_int),
    "t213_server_run_alone": ([_vp, ctypes.POINTER(Request), ctypes.POINTER(ctypes.c_uint64)], ctypes.c_int),
    "t213_server_destroy": ([_vp], ctypes.c_int),
}


def header_functions() -> list[str]:
    """Names of every function declared in include/t213*.h."""
    names = []
    inc = os.path.join(ROOT, "include")
    for f in sorted(os.listdir(inc)):
        if f.startswith("t213") and f.endswith(".h"):
            txt = open(os.path.join(inc, f)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names += re.findall(r"\b(t213_\w+)\s*\(", txt)
    return sorted(set(names))


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(SO_PATH):
            raise ImportError(f"{SO_PATH} is not built; run `python 213transpose_b200/build.py` "
                              "(there is no CPU fallback)")
        L = ctypes.CDLL(SO_PATH)
        for name, (args, res) in _SIGS.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _lib = L
    return _lib


def check(status: int) -> None:
    if status != OK:
        L = lib()
        raise T213Error(status, f"{L.t213_status_string(status).decode()}: {L.t213_last_error().decode()}")


def params(vals) -> ctypes.Array:
    vals = [int(v) for v in vals]
    arr = (ctypes.c_int64 * max(1, len(vals)))(*vals) if vals else (ctypes.c_int64 * 1)(0)
    return arr
