"""ctypes binding of libb200knn.so (C ABI declared in include/b200knn.h).

The library is the only compute path: if it is missing or cannot be loaded,
every call raises ``BackendExecutionError``.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

from .exceptions import BackendExecutionError

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libb200knn.so")

B2K_OK = 0
B2K_EINVAL = 1
B2K_ENONFINITE = 2
B2K_ENOMEM = 3
B2K_ECUDA = 4
B2K_ETIMEOUT = 5
B2K_EUNSUPPORTED = 6
B2K_EINJECTED = 7

MODE_AUTO = 0
MODE_FP32 = 1
MODE_BF16 = 2
MODE_EXACT = 3
MODE_TF32 = 4
MODE_U8 = 5
MODE_SQUARED = 16  # flag: squared distances (B2K_MODE_SQUARED)
MODES = {"auto": MODE_AUTO, "fp32": MODE_FP32, "bf16": MODE_BF16, "exact": MODE_EXACT,
         "tf32": MODE_TF32, "u8": MODE_U8}


class Stats(ctypes.Structure):
    _fields_ = [
        ("mode_used", ctypes.c_int32),
        ("splits", ctypes.c_int32),
        ("candidates", ctypes.c_int64),
        ("list_entries", ctypes.c_int64),
        ("fallback_rows", ctypes.c_int64),
        ("second_pass_rows", ctypes.c_int64),
        ("exact_compares", ctypes.c_int64),
        ("screen_ms", ctypes.c_double),
        ("total_ms", ctypes.c_double),
        ("refined", ctypes.c_int64),
        ("seed_ms", ctypes.c_double),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class Problem(ctypes.Structure):
    """b2k_problem: one kNN problem of a batch (device pointers)."""

    _fields_ = [
        ("index", ctypes.c_void_p),
        ("queries", ctypes.c_void_p),
        ("m", ctypes.c_int64),
        ("k", ctypes.c_int32),
        ("exclude_self", ctypes.c_int32),
        ("q_offset", ctypes.c_int64),
        ("dist", ctypes.c_void_p),
        ("idx", ctypes.c_void_p),
    ]


class BatchStats(ctypes.Structure):
    _fields_ = [
        ("problems", ctypes.c_int32),
        ("graph_problems", ctypes.c_int32),
        ("screen_launches", ctypes.c_int32),
        ("work_items", ctypes.c_int32),
        ("candidates", ctypes.c_int64),
        ("fallback_rows", ctypes.c_int64),
        ("exact_compares", ctypes.c_int64),
        ("tune_ms", ctypes.c_float),
        ("run_ms", ctypes.c_float),
    ]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


BATCH_AUTOTUNE = 1

# Every exported symbol of the C ABI, with (restype, argtypes).
_vp, _i32, _i64, _dbl = ctypes.c_void_p, ctypes.c_int32, ctypes.c_int64, ctypes.c_double
SIGNATURES = {
    "b2k_version": (ctypes.c_int, []),
    "b2k_last_error": (ctypes.c_char_p, []),
    "b2k_index_create": (ctypes.c_int, [_vp, _i64, _i32, _i32, ctypes.POINTER(_vp)]),
    "b2k_index_create_device": (ctypes.c_int, [_vp, _i64, _i32, _vp, ctypes.POINTER(_vp)]),
    "b2k_index_destroy": (ctypes.c_int, [_vp]),
    "b2k_index_shape": (ctypes.c_int, [_vp, ctypes.POINTER(_i64), ctypes.POINTER(_i32)]),
    "b2k_index_download": (ctypes.c_int, [_vp, _vp]),
    "b2k_index_device_data": (_vp, [_vp]),
    "b2k_knn": (ctypes.c_int, [_vp, _vp, _i64, _i32, _i32, _i64, _i32, _vp, _vp,
                               ctypes.POINTER(Stats)]),
    "b2k_knn_device": (ctypes.c_int, [_vp, _vp, _i64, _i32, _i32, _i64, _i32, _vp, _vp, _vp,
                                      ctypes.POINTER(Stats)]),
    "b2k_knn_device_noalloc": (ctypes.c_int, [_vp, _vp, _i64, _i32, _i32, _i64, _vp, _vp,
                                              _vp]),
    "b2k_knn_backward": (ctypes.c_int, [_vp, _i64, _vp, _i64, _i32, _i32, _vp, _vp, _vp, _i32,
                                        _vp, _vp, _vp]),
    "b2k_knn_segments": (ctypes.c_int, [_vp, _vp, _i32, _vp, _vp, _i32, _i32, _i32, _vp, _vp,
                                        _vp]),
    "b2k_class_votes": (ctypes.c_int, [_vp, _vp, _i64, _i32, _vp, _i32, _i32, _vp, _vp, _vp]),
    "b2k_shard_merge": (ctypes.c_int, [_vp, _vp, _i32, _i64, _i32, _i32, _i32, _i64, _vp, _vp,
                                       _vp, _vp]),
    "b2k_shard_keys": (ctypes.c_int, [_vp, _i64, _vp, _vp, _i32, _i64, _i32, _vp, _i64, _vp,
                                      _vp]),
    "b2k_shard_resolve": (ctypes.c_int, [_vp, _vp, _i32, _i64, _i32, _i32, _i64, _vp, _i64, _vp,
                                         _vp, _vp, _vp]),
    "b2k_radius": (ctypes.c_int, [_vp, _vp, _i64, _dbl, _i32, _i64, _i32, _i32,
                                  ctypes.POINTER(_vp)]),
    "b2k_radius_result_nnz": (ctypes.c_int, [_vp, ctypes.POINTER(_i64)]),
    "b2k_radius_result_fetch": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "b2k_radius_result_release": (ctypes.c_int, [_vp]),
    "b2k_radius_result_class_votes": (ctypes.c_int, [_vp, _vp, _i32, _i32, _vp, _vp, _vp]),
    "b2k_radius_result_class_predict": (ctypes.c_int, [_vp, _vp, _i32, _vp, _vp, _vp]),
    "b2k_radius_result_means": (ctypes.c_int, [_vp, _vp, _i32, _vp, _vp, _vp]),
    "b2k_batch_create": (ctypes.c_int, [ctypes.POINTER(Problem), _i32, _i32, _vp,
                                        ctypes.POINTER(_vp)]),
    "b2k_batch_run": (ctypes.c_int, [_vp, _vp]),
    "b2k_batch_finish": (ctypes.c_int, [_vp, _vp, ctypes.POINTER(BatchStats)]),
    "b2k_batch_destroy": (ctypes.c_int, [_vp]),
    "b2k_batch_submit": (ctypes.c_int, [ctypes.POINTER(Problem), _i32, _vp]),
}

_lib = None
_lock = threading.Lock()


def load():
    """Load libb200knn.so once; raise if it is absent (no silent fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(LIB_PATH):
                raise BackendExecutionError(
                    f"{LIB_PATH} is missing: build it with `python -m mlxlearn_b200._build` "
                    "(there is no CPU fallback)")
            lib = ctypes.CDLL(LIB_PATH)
            for name, (res, args) in SIGNATURES.items():
                fn = getattr(lib, name)
                fn.restype = res
                fn.argtypes = args
            _lib = lib
    return _lib


def last_error() -> str:
    msg = load().b2k_last_error()
    return msg.decode() if msg else ""


def check(rc: int, what: str = "") -> None:
    """Map a status code to the exception the reference raises for it."""
    if rc == B2K_OK:
        return
    msg = last_error() or f"{what} failed with status {rc}"
    if rc in (B2K_EINVAL, B2K_ENONFINITE):
        raise ValueError(msg)
    if rc == B2K_ENOMEM:
        raise MemoryError(msg)
    raise BackendExecutionError(msg, status=rc)


def ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data
