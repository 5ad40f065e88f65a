"""ctypes binding of include/bolt_b200.h (the C ABI of libboltb200.so).

Struct layouts here must match the header field for field. The library is
loaded from this directory; a missing library raises instead of falling back
to anything else.
"""

from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libboltb200.so"

# bolt_status
OK, DECLINE, ERR_SPILL, ERR_OVERFLOW, ERR_CAPACITY, ERR_TIMEOUT, ERR_CUDA, ERR_INVALID = range(8)
STATUS_NAMES = ["ok", "decline", "spill", "overflow", "capacity", "timeout", "cuda", "invalid"]

# bolt_dtype
I32, I64, F32, F64, DEC128, U32 = range(6)
DTYPE_CODES = {"i32": I32, "i64": I64, "f32": F32, "f64": F64, "dec128": DEC128, "u32": U32}

# bolt_agg_op
AGG_SUM, AGG_COUNT_STAR, AGG_COUNT, AGG_MIN, AGG_MAX, AGG_AVG = range(6)
AGG_CODES = {"sum": AGG_SUM, "count_star": AGG_COUNT_STAR, "count": AGG_COUNT,
             "min": AGG_MIN, "max": AGG_MAX, "avg": AGG_AVG}

# bolt_cmp
CMP_CODES = {"<": 0, "<=": 1, ">": 2, ">=": 3, "==": 4, "=": 4, "!=": 5, "<>": 5}

FLAG_ASYNC = 0x1
FLAG_PROFILE = 0x2
FLAG_FORCE_GLOBAL = 0x4
FLAG_FORCE_SHMEM = 0x8
FLAG_NO_TUNE = 0x10
FLAG_KERNEL_REGS = 0x20
FLAG_KERNEL_STAGED = 0x40
FLAG_NO_PART = 0x80
FLAG_FORCE_PART = 0x100
FLAG_KERNEL_TIMES = 0x200


class ColView(C.Structure):
    _fields_ = [("data", C.c_void_p), ("validity", C.c_void_p), ("len", C.c_uint64),
                ("dtype", C.c_int32), ("scale", C.c_int32)]


class ColMut(C.Structure):
    _fields_ = [("data", C.c_void_p), ("validity", C.c_void_p), ("cap", C.c_uint64),
                ("dtype", C.c_int32), ("scale", C.c_int32)]


class AggSpec(C.Structure):
    _fields_ = [("op", C.c_int32), ("input_col", C.c_int32)]


class Pred(C.Structure):
    _fields_ = [("col", C.c_int32), ("cmp", C.c_int32), ("lit_i", C.c_int64), ("lit_f", C.c_double)]


class GroupbyDesc(C.Structure):
    _fields_ = [("cols", C.POINTER(ColView)), ("n_cols", C.c_int32),
                ("key_cols", C.POINTER(C.c_int32)), ("n_keys", C.c_int32),
                ("preds", C.POINTER(Pred)), ("n_preds", C.c_int32),
                ("aggs", C.POINTER(AggSpec)), ("n_aggs", C.c_int32),
                ("groups_hint", C.c_uint64)]


class GroupbyOut(C.Structure):
    _fields_ = [("keys", C.POINTER(ColMut)), ("aggs", C.POINTER(ColMut)),
                ("n_groups", C.c_uint64), ("n_groups_dev", C.c_void_p)]


class Query(C.Structure):
    _fields_ = [("desc", GroupbyDesc), ("out", GroupbyOut), ("row_begin", C.c_uint64),
                ("row_end", C.c_uint64), ("status", C.c_int32)]


class ServerConfig(C.Structure):
    _fields_ = [("device", C.c_int32), ("scratch_bytes", C.c_uint64), ("max_batch", C.c_int32),
                ("n_lanes", C.c_int32)]


# name -> (restype, argtypes)
SIGNATURES = {
    "bolt_ctx_create": (C.c_int, [C.c_int, C.c_uint64, C.POINTER(C.c_void_p)]),
    "bolt_ctx_destroy": (None, [C.c_void_p]),
    "bolt_ctx_last_error": (C.c_char_p, [C.c_void_p]),
    "bolt_status_str": (C.c_char_p, [C.c_int]),
    "bolt_ctx_last_device_ms": (C.c_double, [C.c_void_p]),
    "bolt_ctx_last_launches": (C.c_uint32, [C.c_void_p]),
    "bolt_ctx_last_groupby_tier": (C.c_int32, [C.c_void_p]),
    "bolt_ctx_kernel_times": (C.c_uint32, [C.c_void_p, C.POINTER(C.c_double), C.c_uint32]),
    "bolt_ctx_sync_status": (C.c_int, [C.c_void_p, C.c_void_p]),
    "bolt_ctx_scratch_bytes": (C.c_uint64, [C.c_void_p]),
    "bolt_version": (C.c_char_p, []),
    "bolt_groupby": (C.c_int, [C.c_void_p, C.POINTER(GroupbyDesc), C.POINTER(GroupbyOut), C.c_uint32, C.c_void_p]),
    "bolt_groupby_host": (C.c_int, [C.c_void_p, C.POINTER(GroupbyDesc), C.POINTER(GroupbyOut), C.c_uint32,
                                    C.c_void_p]),
    "bolt_groupby_noalloc": (C.c_int, [C.POINTER(GroupbyDesc), C.POINTER(GroupbyOut), C.c_void_p, C.c_char_p,
                                       C.c_int32]),
    "bolt_groupby_autotune": (C.c_int, [C.c_void_p, C.POINTER(GroupbyDesc), C.POINTER(GroupbyOut), C.c_void_p,
                                        C.POINTER(C.c_double)]),
    "bolt_ctx_tuning_save": (C.c_int, [C.c_void_p, C.c_char_p]),
    "bolt_ctx_tuning_load": (C.c_int, [C.c_void_p, C.c_char_p]),
    "bolt_hash_join_build": (C.c_int, [C.c_void_p, C.POINTER(ColView), C.POINTER(ColView), C.c_uint32,
                                       C.c_void_p, C.POINTER(C.c_void_p)]),
    "bolt_hash_join_probe": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(ColView), C.POINTER(ColMut),
                                       C.POINTER(ColMut), C.POINTER(C.c_uint64), C.c_uint32, C.c_void_p]),
    "bolt_hash_join_release": (None, [C.c_void_p, C.c_void_p]),
    "bolt_join_groupby": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(ColView), C.POINTER(ColView),
                                    C.POINTER(ColMut), C.POINTER(ColMut), C.POINTER(ColMut),
                                    C.POINTER(C.c_uint64), C.c_uint32, C.c_void_p]),
    "bolt_radix_sort_perm": (C.c_int, [C.c_void_p, C.POINTER(ColView), C.c_int32, C.c_int32,
                                       C.POINTER(ColMut), C.c_uint32, C.c_void_p]),
    "bolt_radix_sort_perm_multi": (C.c_int, [C.c_void_p, C.POINTER(ColView), C.c_int32, C.POINTER(C.c_int32),
                                             C.POINTER(C.c_int32), C.POINTER(ColMut), C.c_uint32, C.c_void_p]),
    "bolt_compact": (C.c_int, [C.c_void_p, C.POINTER(ColView), C.c_int32, C.POINTER(Pred), C.c_int32,
                               C.POINTER(ColMut), C.POINTER(ColMut), C.POINTER(C.c_uint64), C.c_uint32,
                               C.c_void_p]),
    "bolt_compact_mask": (C.c_int, [C.c_void_p, C.POINTER(ColView), C.c_int32, C.c_void_p, C.POINTER(ColMut),
                                    C.POINTER(ColMut), C.POINTER(C.c_uint64), C.c_uint32, C.c_void_p]),
    "bolt_batch_groupby": (C.c_int, [C.c_void_p, C.POINTER(Query), C.c_int32, C.c_uint32, C.c_void_p]),
    "bolt_groupby_footprint": (C.c_uint64, [C.POINTER(GroupbyDesc), C.c_uint64]),
    "bolt_batch_graph_create": (C.c_int, [C.c_int, C.POINTER(Query), C.c_int32, C.POINTER(C.c_void_p)]),
    "bolt_graph_launch": (C.c_int, [C.c_void_p, C.c_void_p]),
    "bolt_graph_sync_status": (C.c_int, [C.c_void_p, C.c_void_p, C.POINTER(C.c_int32), C.POINTER(C.c_uint64)]),
    "bolt_graph_destroy": (None, [C.c_void_p]),
    "bolt_server_create": (C.c_int, [C.POINTER(ServerConfig), C.POINTER(C.c_void_p)]),
    "bolt_server_submit": (C.c_int, [C.c_void_p, C.POINTER(Query), C.POINTER(C.c_uint64)]),
    "bolt_server_submit_batch": (C.c_int, [C.c_void_p, C.POINTER(Query), C.c_int32, C.POINTER(C.c_uint64)]),
    "bolt_server_wait": (C.c_int, [C.c_void_p, C.c_uint64, C.POINTER(C.c_double)]),
    "bolt_server_destroy": (None, [C.c_void_p]),
}

_LIB = None


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Loads libboltb200.so and declares every entry point's signature."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise FileNotFoundError(
            f"{p} is missing: build it with `python craton-bolt_b200/build.py` "
            "(the GPU operators have no fallback)")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _LIB = lib
    return lib
