"""CPU oracle: ctypes wrapper of oracle/libbolt_oracle.so.

TEST INFRASTRUCTURE ONLY. Imported by tests/, __graft_entry__.smoke() and
bench.py's CPU-baseline / reference legs as the checker; the product library
never loads it. Each function restates the reference's semantics for this
path (see bolt_oracle.c for the file:line it follows).
"""

from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "libbolt_oracle.so"

I32, I64, F32, F64, DEC128, U32 = range(6)
DT = {"i32": I32, "i64": I64, "f32": F32, "f64": F64, "dec128": DEC128, "u32": U32}
OK, DECLINE, OVERFLOW, CAPACITY, INVALID = 0, 1, 3, 4, 7
AGG = {"sum": 0, "count_star": 1, "count": 2, "min": 3, "max": 4, "avg": 5}
CMP = {"<": 0, "<=": 1, ">": 2, ">=": 3, "==": 4, "=": 4, "!=": 5, "<>": 5}


class OrcCol(C.Structure):
    _fields_ = [("data", C.c_void_p), ("validity", C.c_void_p), ("dtype", C.c_int32), ("scale", C.c_int32)]


class OrcPred(C.Structure):
    _fields_ = [("col", C.c_int32), ("cmp", C.c_int32), ("lit_i", C.c_int64), ("lit_f", C.c_double)]


class OrcAgg(C.Structure):
    _fields_ = [("op", C.c_int32), ("input_col", C.c_int32)]


_lib = None


def build() -> Path:
    """Compiles the oracle with its Makefile (gcc)."""
    subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        _lib = C.CDLL(str(LIB))
    return _lib


class OracleError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(message)
        self.status = status


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class HostCol:
    """Host column for the oracle: numpy data (dec128 = (n, 2) int64), optional
    Arrow bitmap (uint8), dtype code."""

    def __init__(self, data: np.ndarray, dtype: str, validity: np.ndarray | None = None, scale: int = 0):
        self.data = np.ascontiguousarray(data)
        self.dtype = dtype
        self.validity = None if validity is None else np.ascontiguousarray(validity, dtype=np.uint8)
        self.scale = scale

    def c(self) -> OrcCol:
        return OrcCol(_ptr(self.data), _ptr(self.validity), DT[self.dtype], self.scale)


def _cols(table: dict):
    names = list(table.keys())
    arr = (OrcCol * len(names))(*[table[k].c() for k in names])
    return names, arr


def host_threads() -> int:
    """Host threads this process may run on."""
    import os

    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


def groupby(table: dict, group_by, aggs, where=(), threads: int = 1):
    """GROUP BY restated from groupby.rs:295-833. Returns dict with 'keys'
    (packed i64), 'key_null', per-aggregate 'vals' / 'valid' and 'accurate'
    (compensated f64 sums), 'n_groups'. `threads` > 1 runs the same fold on
    that many host threads (key-range partitions, each folded in row order):
    identical results."""
    names, arr = _cols(table)
    n = len(table[group_by[0]].data)
    kidx = (C.c_int32 * len(group_by))(*[names.index(k) for k in group_by])
    preds = []
    for cname, cmp, lit in where:
        if table[cname].dtype in ("f32", "f64"):
            preds.append(OrcPred(names.index(cname), CMP[cmp], 0, float(lit)))
        else:
            preds.append(OrcPred(names.index(cname), CMP[cmp], int(lit), 0.0))
    parr = (OrcPred * max(1, len(preds)))(*preds)
    specs = []
    for op, cname in aggs:
        op = op.lower()
        if op == "count" and cname is None:
            op = "count_star"
        specs.append(OrcAgg(AGG[op], names.index(cname) if cname is not None else -1))
    sarr = (OrcAgg * len(specs))(*specs)
    cap = n + 1
    keys = np.zeros(cap, np.int64)
    knull = np.zeros(cap, np.uint8)
    vals, valids, accs = [], [], []
    for (op, cname) in aggs:
        dt = table[cname].dtype if cname is not None else None
        if op.lower() == "sum" and dt == "dec128":
            vals.append(np.zeros((cap, 2), np.int64))
        elif op.lower() in ("avg",) or (dt in ("f32", "f64") and op.lower() in ("sum", "min", "max")):
            vals.append(np.zeros(cap, np.float64))
        else:
            vals.append(np.zeros(cap, np.int64))
        valids.append(np.zeros(cap, np.uint8))
        accs.append(np.zeros(cap, np.float64))
    vptr = (C.c_void_p * len(aggs))(*[v.ctypes.data for v in vals])
    valptr = (C.c_void_p * len(aggs))(*[v.ctypes.data for v in valids])
    accptr = (C.c_void_p * len(aggs))(*[v.ctypes.data for v in accs])
    ng = C.c_uint64(0)
    err = C.create_string_buffer(256)
    args = [C.c_uint64(n), arr, len(names), kidx, len(group_by), parr, len(preds), sarr, len(specs),
            keys.ctypes.data_as(C.c_void_p), knull.ctypes.data_as(C.c_void_p), vptr, valptr, accptr,
            C.c_uint64(cap), C.byref(ng), err, 256]
    if threads > 1:
        f = lib().orc_groupby_par
        args.append(C.c_int32(int(threads)))
    else:
        f = lib().orc_groupby
    f.restype = C.c_int
    st = f(*args)
    if st != OK:
        raise OracleError(st, err.value.decode() or f"oracle status {st}")
    g = int(ng.value)
    return {"keys": keys[:g], "key_null": knull[:g].astype(bool), "vals": [v[:g] for v in vals],
            "valid": [v[:g].astype(bool) for v in valids], "accurate": [a[:g] for a in accs], "n_groups": g}


def hash_join(build_key: HostCol, probe_key: HostCol):
    nb, npr = len(build_key.data), len(probe_key.data)
    op = np.zeros(max(npr, 1), np.uint32)
    ob = np.zeros(max(npr, 1), np.uint32)
    n = C.c_uint64(0)
    f = lib().orc_hash_join
    f.restype = C.c_int
    st = f(C.c_uint64(nb), C.byref(build_key.c()), C.c_uint64(npr), C.byref(probe_key.c()),
           _ptr(op), _ptr(ob), C.c_uint64(npr), C.byref(n))
    if st != OK:
        raise OracleError(st, f"oracle hash join status {st}")
    k = int(n.value)
    return op[:k], ob[:k]


def groupby_wide(table: dict, group_by: list, aggs: list) -> dict:
    """GROUP BY over two integer key columns wider than 64 bits together (the
    reference's host wide-key reduction): keys sorted by (key0, key1); per
    aggregate the values (int64 or float64 by the aggregate's result) and a
    validity flag."""
    k0, k1 = table[group_by[0]], table[group_by[1]]
    n = len(k0.data)
    na = len(aggs)
    ops = np.array([AGG[op] for op, _ in aggs], np.int32)
    ins = (OrcCol * max(na, 1))(*[table[c].c() if c is not None else OrcCol(None, None, 0, 0) for _, c in aggs])
    cap = max(n, 1)
    ok0 = np.zeros(cap, np.int64)
    ok1 = np.zeros(cap, np.int64)
    oi = np.zeros(na * cap, np.int64)
    of = np.zeros(na * cap, np.float64)
    ov = np.zeros(na * cap, np.uint8)
    ng = C.c_uint64(0)
    f = lib().orc_groupby_wide
    f.restype = C.c_int
    st = f(C.c_uint64(n), C.byref(k0.c()), C.byref(k1.c()), C.c_int32(na), _ptr(ops), ins, _ptr(ok0), _ptr(ok1),
           _ptr(oi), _ptr(of), _ptr(ov), C.c_uint64(cap), C.byref(ng))
    if st != OK:
        raise OracleError(st, f"oracle wide GROUP BY status {st}")
    g = int(ng.value)
    vals, valid = [], []
    for a, (op, c) in enumerate(aggs):
        in_dt = table[c].dtype if c is not None else None
        is_f = op == "avg" or (op in ("sum", "min", "max") and in_dt in ("f32", "f64"))
        vals.append((of if is_f else oi)[a * cap: a * cap + g].copy())
        valid.append(ov[a * cap: a * cap + g].astype(bool))
    return {"n_groups": g, "k0": ok0[:g].copy(), "k1": ok1[:g].copy(), "vals": vals, "valid": valid}


def hash_join_multi(build_key: HostCol, probe_key: HostCol, cap: int | None = None):
    """INNER join with any build keys (duplicates included): (probe_row,
    build_row) pairs in probe order, then build-row order."""
    nb, npr = len(build_key.data), len(probe_key.data)
    if cap is None:
        cap = max(npr, 1) * 4
    op = np.zeros(max(cap, 1), np.uint32)
    ob = np.zeros(max(cap, 1), np.uint32)
    n = C.c_uint64(0)
    f = lib().orc_hash_join_multi
    f.restype = C.c_int
    st = f(C.c_uint64(nb), C.byref(build_key.c()), C.c_uint64(npr), C.byref(probe_key.c()),
           _ptr(op), _ptr(ob), C.c_uint64(cap), C.byref(n))
    if st == CAPACITY:
        return hash_join_multi(build_key, probe_key, int(n.value))
    if st != OK:
        raise OracleError(st, f"oracle multi-match hash join status {st}")
    k = int(n.value)
    return op[:k], ob[:k]


def join_groupby(build_key: HostCol, build_payload: np.ndarray, probe_key: HostCol, value: HostCol | None,
                 max_groups: int = 1 << 16):
    g = np.zeros(max_groups, np.int32)
    lo = np.zeros(max_groups, np.int64)
    hi = np.zeros(max_groups, np.int64)
    cnt = np.zeros(max_groups, np.int64)
    ng = C.c_uint64(0)
    err = C.create_string_buffer(256)
    payload = np.ascontiguousarray(build_payload, dtype=np.int32)
    f = lib().orc_join_groupby
    f.restype = C.c_int
    st = f(C.c_uint64(len(build_key.data)), C.byref(build_key.c()), _ptr(payload),
           C.c_uint64(len(probe_key.data)), C.byref(probe_key.c()),
           C.byref(value.c()) if value is not None else None,
           _ptr(g), _ptr(lo), _ptr(hi), _ptr(cnt), C.c_uint64(max_groups), C.byref(ng), err, 256)
    if st != OK:
        raise OracleError(st, err.value.decode() or f"oracle status {st}")
    k = int(ng.value)
    return g[:k], lo[:k], hi[:k], cnt[:k]


def sort_perm(keys, descending=False, nulls_first=False) -> np.ndarray:
    keys = list(keys) if isinstance(keys, (list, tuple)) else [keys]
    nk = len(keys)
    desc = [descending] * nk if isinstance(descending, bool) else list(descending)
    nf = [nulls_first] * nk if isinstance(nulls_first, bool) else list(nulls_first)
    n = len(keys[0].data)
    perm = np.zeros(max(n, 1), np.uint32)
    arr = (OrcCol * nk)(*[k.c() for k in keys])
    f = lib().orc_sort_perm_multi
    f.restype = C.c_int
    f(C.c_uint64(n), arr, nk, (C.c_int32 * nk)(*map(int, desc)), (C.c_int32 * nk)(*map(int, nf)), _ptr(perm))
    return perm[:n]


def sort_keys(key: HostCol, descending=False) -> np.ndarray:
    """The radix sort key of every row (gpu_sort.rs:1089-1163)."""
    f = lib().orc_sort_key
    f.restype = C.c_uint64
    c = key.c()
    return np.array([f(C.byref(c), C.c_uint64(i), int(descending)) for i in range(len(key.data))], np.uint64)


def compact(table: dict, where=()) -> np.ndarray:
    names, arr = _cols(table)
    n = len(table[names[0]].data)
    preds = []
    for cname, cmp, lit in where:
        if table[cname].dtype in ("f32", "f64"):
            preds.append(OrcPred(names.index(cname), CMP[cmp], 0, float(lit)))
        else:
            preds.append(OrcPred(names.index(cname), CMP[cmp], int(lit), 0.0))
    parr = (OrcPred * max(1, len(preds)))(*preds)
    rows = np.zeros(max(n, 1), np.uint32)
    k = C.c_uint64(0)
    f = lib().orc_compact
    f.restype = C.c_int
    f(C.c_uint64(n), arr, parr, len(preds), _ptr(rows), C.byref(k))
    return rows[: int(k.value)]


def xorshift64star(seed: int, n: int) -> np.ndarray:
    out = np.zeros(n, np.uint64)
    lib().orc_xorshift64star_fill(C.c_uint64(seed), _ptr(out), C.c_uint64(n))
    return out


def shuffle_deterministic(xs: np.ndarray, seed: int) -> np.ndarray:
    a = np.ascontiguousarray(xs, dtype=np.uint32).copy()
    lib().orc_shuffle_deterministic_u32(_ptr(a), C.c_uint64(len(a)), C.c_uint64(seed))
    return a
