"""Loads libbfgt_b200.so (built in-tree) and declares its C ABI (include/bfgt.h).

There is no fallback: if the library is missing and cannot be built, importing
this module raises.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

from . import build as _build

_lib = None

_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_ip = C.POINTER(C.c_int)
_dp = C.POINTER(C.c_double)

BFGT_OK = 0
BFGT_PREC_FP64 = 0
BFGT_PREC_SPLIT = 1

STATUS = {0: "OK", 1: "ERR_ARG", 2: "ERR_TREE", 3: "ERR_CAPACITY", 4: "ERR_OOM", 5: "ERR_CUDA", 6: "ERR_NODEVICE",
          7: "ERR_TIMEOUT"}


class BfgtError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


def lib_path() -> Path:
    return _build.LIB


def lib():
    global _lib
    if _lib is not None:
        return _lib
    if os.environ.get("BFGT_NO_BUILD"):
        path = _build.LIB
        if not path.exists():
            raise ImportError(f"{path} is missing and BFGT_NO_BUILD is set")
    else:
        path = _build.build()
    L = C.CDLL(str(path))
    L.bfgt_last_error.restype = C.c_char_p
    L.boxfgt_.restype = None
    L.boxfgt_.argtypes = [_ip, _ip, _dp, _dp, _ip, _ip, _ip, _ip, _ip, _ip, _ip, _i32p, _i32p, _f64p, _f64p, _f64p,
                          _ip, _f64p, C.c_void_p, C.c_void_p, _ip, _ip, C.c_void_p, _ip, C.c_void_p, C.c_void_p,
                          C.c_void_p, _f64p]
    L.bfgt_boxfgt.restype = C.c_int
    L.bfgt_boxfgt.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                              _i32p, _i32p, _f64p, _f64p, _f64p, _f64p, C.c_void_p, C.c_int]
    L.bfgt_set_default_precision.restype = C.c_int
    L.bfgt_set_default_precision.argtypes = [C.c_int]
    L.bfgt_plan_cache_clear.restype = C.c_int
    L.bfgt_plan_cache_clear.argtypes = []
    L.bfgt_plan_cache_info.restype = C.c_int
    L.bfgt_plan_cache_info.argtypes = [C.c_void_p]
    L.bfgt_boxfgt_last_bytes.restype = C.c_int
    L.bfgt_boxfgt_last_bytes.argtypes = [C.c_void_p]
    L.bfgt_plan_create.restype = C.c_int
    L.bfgt_plan_create.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int,
                                   C.c_int, C.c_int, C.c_int, _i32p, _i32p, _f64p, _f64p, C.c_int]
    L.bfgt_plan_execute.restype = C.c_int
    L.bfgt_plan_execute.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.bfgt_plan_execute_host.restype = C.c_int
    L.bfgt_plan_execute_host.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.bfgt_plan_graph_capture.restype = C.c_int
    L.bfgt_plan_graph_capture.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.bfgt_plan_graph_launch.restype = C.c_int
    L.bfgt_plan_graph_launch.argtypes = [C.c_void_p, C.c_void_p]
    L.bfgt_plan_stage_ms.restype = C.c_int
    L.bfgt_plan_stage_ms.argtypes = [C.c_void_p, _f64p]
    L.bfgt_plan_reserve_events.restype = C.c_int
    L.bfgt_plan_reserve_events.argtypes = [C.c_void_p, C.c_int]
    L.bfgt_plan_info.restype = C.c_int
    L.bfgt_plan_info.argtypes = [C.c_void_p, _i32p]
    L.bfgt_plan_work.restype = C.c_int
    L.bfgt_plan_work.argtypes = [C.c_void_p, _f64p]
    L.bfgt_plan_execute_pgh.restype = C.c_int
    L.bfgt_plan_execute_pgh.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 5
    L.bfgt_plan_execute_pgh_host.restype = C.c_int
    L.bfgt_plan_execute_pgh_host.argtypes = [C.c_void_p, C.c_int] + [C.c_void_p] * 5
    L.bfgt_plan_eval_targets.restype = C.c_int
    L.bfgt_plan_eval_targets.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
    L.bfgt_plan_execute_adjoint.restype = C.c_int
    L.bfgt_plan_execute_adjoint.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.bfgt_plan_execute_adjoint_host.restype = C.c_int
    L.bfgt_plan_execute_adjoint_host.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.bfgt_plan_execute_noalloc.restype = C.c_int
    L.bfgt_plan_execute_noalloc.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    L.bfgt_noalloc_scratch_bytes.restype = C.c_int
    L.bfgt_noalloc_scratch_bytes.argtypes = [C.POINTER(C.c_size_t)]
    L.bfgt_plan_noalloc_need.restype = C.c_int
    L.bfgt_plan_noalloc_need.argtypes = [C.c_void_p, C.POINTER(C.c_size_t)]
    L.bfgt_plan_autotune.restype = C.c_int
    L.bfgt_plan_autotune.argtypes = [C.c_void_p, C.c_void_p, _f64p]
    L.bfgt_plan_check.restype = C.c_int
    L.bfgt_plan_check.argtypes = [C.c_void_p]
    L.bfgt_plan_set_wait_limit.restype = C.c_int
    L.bfgt_plan_set_wait_limit.argtypes = [C.c_void_p, C.c_uint]
    L.bfgt_plan_destroy.restype = C.c_int
    L.bfgt_plan_destroy.argtypes = [C.c_void_p]
    for name, args in (("bfgt_batch_create", [C.POINTER(C.c_void_p), C.c_int, C.c_void_p]),
                       ("bfgt_batch_layout", [C.c_void_p, C.c_void_p]),
                       ("bfgt_batch_execute", [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
                       ("bfgt_batch_execute_adjoint", [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
                       ("bfgt_batch_graph_capture", [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]),
                       ("bfgt_batch_graph_launch", [C.c_void_p, C.c_void_p]),
                       ("bfgt_batch_stage_ms", [C.c_void_p, _f64p]),
                       ("bfgt_batch_info", [C.c_void_p, _i32p]),
                       ("bfgt_batch_check", [C.c_void_p]),
                       ("bfgt_batch_destroy", [C.c_void_p])):
        f = getattr(L, name)
        f.restype = C.c_int
        f.argtypes = args
    L.bfgt_host_plan_dump.restype = C.c_int
    L.bfgt_host_plan_dump.argtypes = [C.c_int, C.c_double, C.c_double, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                      C.c_int, _i32p, _i32p, _f64p, _f64p] + [C.c_void_p] * 4 + [C.c_int] + \
                                     [C.c_void_p] * 6
    L.bfgt_tree_build_gauss.restype = C.c_int
    L.bfgt_tree_build_gauss.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_double, C.c_double, C.c_int,
                                        C.c_double, C.c_int, _f64p, C.c_int, C.c_int]
    L.bfgt_tree_build_uniform.restype = C.c_int
    L.bfgt_tree_build_uniform.argtypes = [C.POINTER(C.c_void_p), C.c_int, C.c_int, C.c_double, C.c_int, C.c_int,
                                          C.c_int, _f64p]
    L.bfgt_tree_sizes.restype = C.c_int
    L.bfgt_tree_sizes.argtypes = [C.c_void_p, _ip, _ip, _ip]
    L.bfgt_tree_export.restype = C.c_int
    L.bfgt_tree_export.argtypes = [C.c_void_p, _i32p, _i32p, _f64p, _f64p, _f64p]
    L.bfgt_tree_free.restype = C.c_int
    L.bfgt_tree_free.argtypes = [C.c_void_p]
    _lib = L
    return L


def check(rc):
    if rc != BFGT_OK:
        raise BfgtError(rc, lib().bfgt_last_error().decode())
    return rc


def last_error() -> str:
    return lib().bfgt_last_error().decode()
