"""ctypes binding of lib/libzuikaku.so (the C ABI declared in include/zuikaku.h).

There is no fallback: if the library is missing or fails to load, every call
raises.  Build it with ``python -m zuikakucfd_b200.build``.
"""
from __future__ import annotations

import ctypes as C
import threading
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libzuikaku.so"

ZK_OK = 0
ERRORS = {1: "ZK_ERR_ARG", 2: "ZK_ERR_STATE", 3: "ZK_ERR_CUDA", 4: "ZK_ERR_NUMERIC",
          5: "ZK_ERR_UNSUPPORTED", 6: "ZK_ERR_IO", 7: "ZK_ERR_TIMEOUT"}

METHOD = {"weno": 0, "dg": 1}
PRECISION = {"fp64": 0, "mixed": 1, "fp64_fma": 2}
LIMITER = {"reference": 0, "none": 1, "tvb": 2, "tvb_mlp": 3}
FLUX = {"hllc": 0, "hll": 1}
BOUNDARY = {"exchange": 0, "periodic": 1}
RECON = {"weno5": 0, "muscl_minmod": 1, "muscl_vanleer": 2, "muscl_superbee": 3}
MLP_NPARAM = 3457
MLP_IN = 40


class ZkError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class zk_options(C.Structure):
    _fields_ = [("method", C.c_int), ("order", C.c_int), ("precision", C.c_int),
                ("limiter", C.c_int), ("flux", C.c_int), ("boundary", C.c_int),
                ("device", C.c_int), ("tvb_M", C.c_double), ("recon", C.c_int), ("tile_tpc", C.c_int)]


class zk_batch_options(C.Structure):
    _fields_ = [("device", C.c_int), ("policy", C.c_int), ("active_cells", C.c_double),
                ("graph_steps", C.c_int), ("autotune", C.c_int), ("arena_bytes", C.c_size_t),
                ("weno_variant", C.c_int), ("dg_variant", C.c_int)]


class zk_batch_report(C.Structure):
    _fields_ = [("ms", C.c_double), ("cell_updates", C.c_double), ("dof_updates", C.c_double),
                ("latency_p50_ms", C.c_double), ("latency_p99_ms", C.c_double),
                ("latency_max_ms", C.c_double), ("problems", C.c_int), ("done", C.c_int),
                ("failed", C.c_int), ("graph_launches", C.c_int), ("graph_steps", C.c_int),
                ("kernel_launches", C.c_longlong)]


class zk_batch_problem(C.Structure):
    _fields_ = [("state", C.c_int), ("steps_done", C.c_int), ("t", C.c_double),
                ("latency_ms", C.c_double), ("status", C.c_uint32), ("group", C.c_int)]


POLICY = {"all": 0, "sjf": 1}
BATCH_STATE = {0: "waiting", 1: "running", 2: "done", 3: "failed"}

_lock = threading.Lock()
_lib: C.CDLL | None = None

_P = C.c_void_p
_D = C.POINTER(C.c_double)
_SIGS = {
    "zk_default_options": (None, [C.POINTER(zk_options)]),
    "zk_create": (C.c_int, [C.POINTER(zk_options), C.POINTER(_P)]),
    "zk_destroy": (C.c_int, [_P]),
    "zk_last_error": (C.c_char_p, []),
    "zk_version": (C.c_int, []),
    "zk_set_mesh": (C.c_int, [_P, C.c_int, C.c_int, C.c_double, C.c_double, C.POINTER(C.c_int32)]),
    "zk_set_state": (C.c_int, [_P, _D]),
    "zk_get_state": (C.c_int, [_P, _D]),
    "zk_state_size": (C.c_size_t, [_P]),
    "zk_load_case": (C.c_int, [_P, C.c_char_p]),
    "zk_step": (C.c_int, [_P, C.c_double, C.c_int]),
    "zk_rhs": (C.c_int, [_P, C.c_double, _D]),
    "zk_limit": (C.c_int, [_P]),
    "zk_max_speed": (C.c_int, [_P, _D]),
    "zk_recover_primitives": (C.c_int, [_P, _D]),
    "zk_status_word": (C.c_int, [_P, C.POINTER(C.c_uint32)]),
    "zk_set_stream": (C.c_int, [_P, _P]),
    "zk_synchronize": (C.c_int, [_P]),
    "zk_step_timed": (C.c_int, [_P, C.c_double, C.c_int, C.POINTER(C.c_float)]),
    "zk_state_device": (C.c_int, [_P, C.POINTER(_D), C.POINTER(C.c_int)]),
    "zk_peak_flops": (C.c_int, [C.c_int, C.c_int, _D]),
    "zk_set_indicator": (C.c_int, [_P, C.POINTER(C.c_float), C.c_int]),
    "zk_indicator_features": (C.c_int, [_P, C.POINTER(C.c_float), C.POINTER(C.c_uint8)]),
    "zk_limited_cells": (C.c_int, [_P, C.POINTER(C.c_uint32)]),
    "zk_indicator_logits": (C.c_int, [_P, C.POINTER(C.c_float)]),
    "zk_set_indicator_screen": (C.c_int, [_P, C.c_float]),
    "zk_tile_tpc": (C.c_int, [_P, C.POINTER(C.c_int)]),
    "zk_selftest_tma_timeout": (C.c_int, [_P, C.c_uint32, C.POINTER(C.c_uint32)]),
    "zk_indicator_stage_features": (C.c_int, [_P, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_uint8)]),
    "zk_indicator_stage_logits": (C.c_int, [_P, C.c_double, C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                            C.POINTER(C.c_uint32)]),
    "zk_mlp_train": (C.c_int, [C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_uint8), C.c_int64,
                               C.POINTER(C.c_float), C.c_int, C.c_int, C.c_float, C.c_float, C.c_uint64,
                               C.POINTER(C.c_float)]),
    "zk_mlp_grad": (C.c_int, [C.c_int, C.POINTER(C.c_float), C.POINTER(C.c_uint8), C.c_int64,
                              C.POINTER(C.c_float), C.c_float, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "zk_mlp_forward": (C.c_int, [C.c_int, C.POINTER(C.c_float), C.c_int64, C.POINTER(C.c_float), C.c_int,
                                 C.POINTER(C.c_float)]),
    "zk_weno_step_noalloc": (C.c_int, [_D, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double,
                                       C.POINTER(C.c_int32), C.c_double, C.c_int, _P,
                                       C.POINTER(C.c_uint32)]),
    "zk_mach_number": (C.c_int, [_P, _D, _D]),
    "zk_stage": (C.c_int, [_P, C.c_double, C.c_int]),
    "zk_stage_limit": (C.c_int, [_P, C.c_int]),
    "zk_halo_bytes": (C.c_int, [_P, C.c_int, C.POINTER(C.c_size_t)]),
    "zk_halo_pack": (C.c_int, [_P, C.c_int, C.c_int, _P]),
    "zk_halo_unpack": (C.c_int, [_P, C.c_int, C.c_int, _P]),
    "zk_batch_default_options": (None, [C.POINTER(zk_batch_options)]),
    "zk_batch_create": (C.c_int, [C.POINTER(zk_batch_options), C.POINTER(_P)]),
    "zk_batch_add": (C.c_int, [_P, C.POINTER(zk_options), C.c_int, C.c_int, C.c_double, C.c_double,
                               C.POINTER(C.c_int32), _D, C.c_int, C.c_double, C.POINTER(C.c_int)]),
    "zk_batch_run": (C.c_int, [_P, C.POINTER(zk_batch_report)]),
    "zk_batch_get_state": (C.c_int, [_P, C.c_int, _D]),
    "zk_batch_problem_info": (C.c_int, [_P, C.c_int, C.POINTER(zk_batch_problem)]),
    "zk_batch_dt_history": (C.c_int, [_P, C.c_int, _D, C.c_int]),
    "zk_batch_group_config": (C.c_int, [_P, C.c_int] + [C.POINTER(C.c_int)] * 6),
    "zk_batch_group_tile": (C.c_int, [_P, C.c_int] + [C.POINTER(C.c_int)] * 3),
    "zk_batch_destroy": (None, [_P]),
}


def lib() -> C.CDLL:
    """Load the native library once; raise if it is absent."""
    global _lib
    with _lock:
        if _lib is None:
            if not LIB_PATH.exists():
                raise RuntimeError(
                    f"{LIB_PATH} is missing: build it with `python -m zuikakucfd_b200.build` "
                    "(there is no CPU fallback)")
            l = C.CDLL(str(LIB_PATH))
            for name, (res, args) in _SIGS.items():
                f = getattr(l, name)
                f.restype = res
                f.argtypes = args
            _lib = l
    return _lib


def exported_symbols() -> list[str]:
    return list(_SIGS)


def check(rc: int) -> None:
    if rc != ZK_OK:
        raise ZkError(rc, (lib().zk_last_error() or b"").decode(errors="replace"))


def dptr(a) -> "C._Pointer":
    return a.ctypes.data_as(_D)
