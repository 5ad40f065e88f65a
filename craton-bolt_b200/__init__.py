"""bolt-b200: B200-native GROUP BY / hash join / ORDER BY / filter compaction.

Host-side mirror of the Craton Bolt operator interface for this path. The
reference's executors return ``Option<BoltResult<RecordBatch>>``
(src/exec/groupby_shmem_exec.rs:53, src/exec/groupby_tier2_exec.rs:30):
``None`` declines so the caller tries its next path, ``Err`` is a typed
``BoltError`` (src/error.rs:21-100). Here ``try_*`` methods return ``None``
on a decline and every method raises a :class:`BoltError` subclass on an
error; the work itself runs in libboltb200.so through its C ABI.

Columns are :class:`Column` objects over torch tensors. CUDA tensors are used
in place (the reference's GpuView borrow); host tensors / numpy arrays are
copied to the device and results copied back (the end-to-end path).
"""

from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Iterable, Sequence

import numpy as np
import torch

from . import _abi
from ._abi import (AGG_CODES, CMP_CODES, DTYPE_CODES, FLAG_ASYNC, FLAG_FORCE_GLOBAL, FLAG_FORCE_PART,
                   FLAG_FORCE_SHMEM, FLAG_KERNEL_REGS, FLAG_KERNEL_STAGED, FLAG_KERNEL_TIMES, FLAG_NO_PART, FLAG_NO_TUNE,
                   FLAG_PROFILE)

__all__ = ["BoltError", "DeclineError", "SpillError", "TypeError_", "GpuCapacityError", "TimeoutError_",
           "CudaError", "PlanError", "Column", "Engine", "col", "GroupbyResult", "FLAG_ASYNC",
           "FLAG_PROFILE", "FLAG_FORCE_GLOBAL", "FLAG_FORCE_SHMEM", "FLAG_NO_TUNE", "FLAG_KERNEL_REGS",
           "FLAG_KERNEL_STAGED", "FLAG_KERNEL_TIMES", "FLAG_NO_PART", "FLAG_FORCE_PART", "lib", "PreparedGroupby",
           "Server", "BatchGraph"]


# ---------------------------------------------------------------------------
# Errors (the reference's BoltError variants, src/error.rs:21-100)
# ---------------------------------------------------------------------------
class BoltError(RuntimeError):
    status = -1

    def __init__(self, message: str, status: int | None = None):
        super().__init__(message)
        if status is not None:
            self.status = status


class DeclineError(BoltError):
    status = _abi.DECLINE


class SpillError(BoltError):
    """The reference's soft miss: messages start with "partition_reduce spill:"."""
    status = _abi.ERR_SPILL


class TypeError_(BoltError):
    """BoltError::Type — SUM(integer) / SUM(Decimal128) overflow."""
    status = _abi.ERR_OVERFLOW


class GpuCapacityError(BoltError):
    status = _abi.ERR_CAPACITY


class TimeoutError_(BoltError):
    status = _abi.ERR_TIMEOUT


class CudaError(BoltError):
    status = _abi.ERR_CUDA


class PlanError(BoltError):
    status = _abi.ERR_INVALID


_ERRORS = {_abi.DECLINE: DeclineError, _abi.ERR_SPILL: SpillError, _abi.ERR_OVERFLOW: TypeError_,
           _abi.ERR_CAPACITY: GpuCapacityError, _abi.ERR_TIMEOUT: TimeoutError_, _abi.ERR_CUDA: CudaError,
           _abi.ERR_INVALID: PlanError}


def lib() -> C.CDLL:
    return _abi.load()


# ---------------------------------------------------------------------------
# Columns
# ---------------------------------------------------------------------------
_TORCH_DT = {"i32": torch.int32, "i64": torch.int64, "f32": torch.float32, "f64": torch.float64,
             "u32": torch.int32, "dec128": torch.int64}
_NP_DT = {"i32": np.int32, "i64": np.int64, "f32": np.float32, "f64": np.float64, "u32": np.uint32,
          "dec128": np.int64}
_INFER = {np.dtype(np.int32): "i32", np.dtype(np.int64): "i64", np.dtype(np.float32): "f32",
          np.dtype(np.float64): "f64", np.dtype(np.uint32): "u32"}
_INFER_T = {torch.int32: "i32", torch.int64: "i64", torch.float32: "f32", torch.float64: "f64"}


@dataclass
class Column:
    """A column: ``data`` (1-D, or (n, 2) int64 lo/hi words for dec128),
    optional Arrow LSB validity bitmap (uint8), dtype code and decimal scale."""

    data: torch.Tensor
    dtype: str
    validity: torch.Tensor | None = None
    scale: int = 0

    def __len__(self) -> int:
        return int(self.data.shape[0])

    @property
    def is_cuda(self) -> bool:
        return self.data.is_cuda

    def to(self, device, non_blocking: bool = False) -> "Column":
        v = self.validity.to(device, non_blocking=non_blocking) if self.validity is not None else None
        return Column(self.data.to(device, non_blocking=non_blocking), self.dtype, v, self.scale)

    def numpy(self) -> np.ndarray:
        a = self.data.cpu().numpy()
        if self.dtype == "u32":
            return a.view(np.uint32)
        return a

    def valid_mask(self) -> np.ndarray:
        """Boolean per-row validity (all True without a bitmap)."""
        n = len(self)
        if self.validity is None:
            return np.ones(n, dtype=bool)
        bits = np.unpackbits(self.validity.cpu().numpy(), bitorder="little")[:n]
        return bits.astype(bool)

    def view(self) -> _abi.ColView:
        return _abi.ColView(self.data.data_ptr(), self.validity.data_ptr() if self.validity is not None else None,
                            len(self), DTYPE_CODES[self.dtype], self.scale)


def col(values, dtype: str | None = None, validity=None, scale: int = 0) -> Column:
    """Builds a Column from numpy / torch / a Python list. ``validity`` may be a
    boolean mask (True = valid) or an Arrow bitmap (uint8)."""
    if isinstance(values, torch.Tensor):
        t = values
        dt = dtype or _INFER_T[t.dtype]
    else:
        a = np.asarray(values)
        if dtype is None:
            dtype = _INFER[a.dtype]
        a = a.astype(_NP_DT[dtype], copy=False)
        if dtype == "u32":
            a = a.view(np.int32)
        if dtype == "dec128" and a.ndim == 1:
            lo = a.astype(np.int64)
            a = np.stack([lo, np.where(lo < 0, -1, 0).astype(np.int64)], axis=1)
        t = torch.from_numpy(np.ascontiguousarray(a))
        dt = dtype
    v = None
    if validity is not None:
        va = validity.cpu().numpy() if isinstance(validity, torch.Tensor) else np.asarray(validity)
        if va.dtype == bool:
            va = np.packbits(va.astype(np.uint8), bitorder="little")
        v = torch.from_numpy(np.ascontiguousarray(va.astype(np.uint8)))
        if t.is_cuda:
            v = v.to(t.device)
    return Column(t, dt, v, scale)


def _bitmap_bytes(n: int) -> int:
    return (n + 7) // 8 + 8


@dataclass
class GroupbyResult:
    keys: list[Column]
    aggs: list[Column]
    n_groups: int
    device_ms: float = 0.0
    launches: int = 0


_SUM_OUT = {"i32": "i64", "i64": "i64", "f64": "f64", "dec128": "dec128"}


def _agg_out_dtype(op: str, in_dtype: str | None) -> str:
    if op in ("count", "count_star"):
        return "i64"
    if op == "avg":
        return "f64"
    if op == "sum":
        return _SUM_OUT.get(in_dtype, in_dtype)
    return in_dtype


# ---------------------------------------------------------------------------
# Engine
# ---------------------------------------------------------------------------
class Engine:
    """One bolt_ctx (scratch arena + status word) bound to a device and the
    current torch stream of that device. Not thread-safe, like the
    reference's Engine (src/exec/launch.rs:84-100)."""

    def __init__(self, device: int = 0, scratch_bytes: int = 0):
        self._lib = lib()
        self.device = device
        torch.cuda.init()
        h = C.c_void_p()
        st = self._lib.bolt_ctx_create(device, scratch_bytes, C.byref(h))
        if st != _abi.OK:
            raise _ERRORS.get(st, BoltError)(f"bolt_ctx_create failed: {_abi.STATUS_NAMES[st]}", st)
        self._ctx = h
        self.last_device_ms = 0.0
        self.last_launches = 0

    def close(self):
        if getattr(self, "_ctx", None):
            self._lib.bolt_ctx_destroy(self._ctx)
            self._ctx = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def stream_handle(self) -> int:
        return torch.cuda.current_stream(self.device).cuda_stream

    @property
    def last_groupby_tier(self) -> int:
        """Tier of the last GROUP BY: 1 shared-memory + global hash table,
        2 hash-partitioned, 3 the sort-based path for keys wider than 64 bits."""
        return int(self._lib.bolt_ctx_last_groupby_tier(self._ctx))

    @property
    def scratch_bytes(self) -> int:
        return int(self._lib.bolt_ctx_scratch_bytes(self._ctx))

    def _check(self, st: int, what: str, decline_ok: bool = False):
        self.last_device_ms = float(self._lib.bolt_ctx_last_device_ms(self._ctx))
        self.last_launches = int(self._lib.bolt_ctx_last_launches(self._ctx))
        if st == _abi.OK:
            return True
        msg = self._lib.bolt_ctx_last_error(self._ctx).decode() or _abi.STATUS_NAMES[st]
        if st == _abi.DECLINE and decline_ok:
            return False
        raise _ERRORS.get(st, BoltError)(f"{what}: {msg}", st)

    def _dev(self, c: Column) -> Column:
        if c.is_cuda:
            return c
        dev = f"cuda:{self.device}"
        d = c.data if c.data.is_pinned() else c.data.pin_memory()
        v = c.validity.to(dev, non_blocking=True) if c.validity is not None else None
        return Column(d.to(dev, non_blocking=True), c.dtype, v, c.scale)

    def _alloc(self, dtype: str, n: int, with_validity: bool) -> Column:
        shape = (max(n, 1), 2) if dtype == "dec128" else (max(n, 1),)
        t = torch.empty(shape, dtype=_TORCH_DT[dtype], device=f"cuda:{self.device}")
        v = torch.zeros(_bitmap_bytes(n), dtype=torch.uint8, device=f"cuda:{self.device}") if with_validity else None
        return Column(t, dtype, v)

    # ---- GROUP BY -------------------------------------------------------------
    def prepare_groupby(self, table: dict, group_by: Sequence[str], aggs: Sequence[tuple],
                        where: Iterable[tuple] = (), groups_hint: int = 0, out_cap: int | None = None,
                        rows: tuple[int, int] | None = None) -> "PreparedGroupby":
        """Builds the C-ABI descriptor and output columns of one GROUP BY
        (used by execute_groupby, execute_batch and Server.submit)."""
        cols = {k: self._dev(v) for k, v in table.items()}
        return PreparedGroupby(self, cols, list(group_by), list(aggs), list(where), int(groups_hint), out_cap, rows)

    def try_execute_groupby(self, table: dict, group_by: Sequence[str], aggs: Sequence[tuple],
                            where: Iterable[tuple] = (), groups_hint: int = 0, flags: int = 0,
                            out_cap: int | None = None) -> GroupbyResult | None:
        """GROUP BY over ``table`` (name -> Column). ``aggs`` holds
        (op, column name or None) with op in sum/count/count_star/min/max/avg;
        ``where`` holds (column, cmp, literal) conjuncts. Returns None when the
        shape is declined (the reference's ``Ok(None)``)."""
        host_out = not all(v.is_cuda for v in table.values())
        host_in = not any(v.is_cuda for v in table.values())
        if host_in:
            # All columns on the host: stream them through bolt_groupby_host
            # (chunked upload overlapped with the aggregation).
            pq = PreparedGroupby(self, dict(table), list(group_by), list(aggs), list(where), int(groups_hint),
                                 out_cap, None)
            r = self._run_groupby(self._lib.bolt_groupby_host, pq, flags, host_out, "GROUP BY (host columns)")
            if r is not None or "row-order overflow check" not in self._lib.bolt_ctx_last_error(self._ctx).decode():
                return r
        pq = self.prepare_groupby(table, group_by, aggs, where, groups_hint, out_cap)
        return self._run_groupby(self._lib.bolt_groupby, pq, flags, host_out, "GROUP BY")

    def _run_groupby(self, fn, pq: "PreparedGroupby", flags: int, host_out: bool, what: str):
        for _attempt in range(2):
            st = fn(self._ctx, C.byref(pq.desc), C.byref(pq.out), flags | FLAG_PROFILE, C.c_void_p(self.stream_handle))
            if st == _abi.ERR_CAPACITY and pq.out.n_groups > pq.cap:
                pq.realloc(int(pq.out.n_groups))
                continue
            if not self._check(st, what, decline_ok=True):
                return None
            self._lib.bolt_ctx_kernel_times(self._ctx, None, 1 << 20)
            return pq.result(host_out)
        raise GpuCapacityError(f"{what}: output capacity retry failed", _abi.ERR_CAPACITY)

    def execute_groupby(self, *args, **kw) -> GroupbyResult:
        r = self.try_execute_groupby(*args, **kw)
        if r is None:
            raise DeclineError(f"GROUP BY declined: {self._lib.bolt_ctx_last_error(self._ctx).decode()}")
        return r

    def autotune_groupby(self, pq: "PreparedGroupby") -> float:
        """Times candidate launch choices for this query shape on the device
        and keeps the fastest in the context (bolt_groupby_autotune).
        Returns the winner's device milliseconds."""
        best = C.c_double(0.0)
        st = self._lib.bolt_groupby_autotune(self._ctx, C.byref(pq.desc), C.byref(pq.out),
                                             C.c_void_p(self.stream_handle), C.byref(best))
        self._check(st, "GROUP BY autotune")
        return float(best.value)

    def save_tuning(self, path: str):
        if self._lib.bolt_ctx_tuning_save(self._ctx, str(path).encode()) != _abi.OK:
            raise PlanError(f"cannot write tuning file {path}")

    def load_tuning(self, path: str):
        st = self._lib.bolt_ctx_tuning_load(self._ctx, str(path).encode())
        self._check(st, "load tuning")

    def execute_batch(self, prepared: Sequence["PreparedGroupby"], flags: int = 0) -> list[GroupbyResult]:
        """Runs many prepared GROUP BY queries as one batch (one persistent
        aggregation launch + one batched finalize)."""
        qs = (_abi.Query * len(prepared))(*[pq.query() for pq in prepared])
        st = self._lib.bolt_batch_groupby(self._ctx, qs, len(prepared), flags, C.c_void_p(self.stream_handle))
        self._check(st, "batched GROUP BY")
        out = []
        for pq, q in zip(prepared, qs):
            pq.out.n_groups = q.out.n_groups
            out.append(pq.result(False))
        return out


    @staticmethod
    def _mut(c: Column, cap: int) -> _abi.ColMut:
        return _abi.ColMut(c.data.data_ptr(), c.validity.data_ptr() if c.validity is not None else None, cap,
                           DTYPE_CODES[c.dtype], c.scale)

    @staticmethod
    def _trim(c: Column, n: int) -> Column:
        v = c.validity[: (n + 7) // 8] if c.validity is not None else None
        return Column(c.data[:n], c.dtype, v, c.scale)

    # ---- ORDER BY -------------------------------------------------------------
    def sort_indices(self, keys: Sequence[Column], descending: Sequence[bool] | bool = False,
                     nulls_first: Sequence[bool] | bool = False, flags: int = 0) -> torch.Tensor:
        """Stable ORDER BY permutation (u32 stored in an int32 tensor)."""
        keys = [self._dev(k) for k in keys]
        nk = len(keys)
        desc = [descending] * nk if isinstance(descending, bool) else list(descending)
        nf = [nulls_first] * nk if isinstance(nulls_first, bool) else list(nulls_first)
        n = len(keys[0])
        perm = torch.empty(max(n, 1), dtype=torch.int32, device=f"cuda:{self.device}")
        views = (_abi.ColView * nk)(*[k.view() for k in keys])
        pm = _abi.ColMut(perm.data_ptr(), None, n, _abi.U32, 0)
        st = self._lib.bolt_radix_sort_perm_multi(self._ctx, views, nk, (C.c_int32 * nk)(*map(int, desc)),
                                                  (C.c_int32 * nk)(*map(int, nf)), C.byref(pm),
                                                  flags | FLAG_PROFILE, C.c_void_p(self.stream_handle))
        self._check(st, "ORDER BY")
        return perm[:n]

    # ---- filter compaction ------------------------------------------------------
    def compact_columns(self, table: dict, where: Iterable[tuple] = (), mask: torch.Tensor | None = None,
                        out_cap: int | None = None, flags: int = 0, with_row_ids: bool = True):
        """Order-preserving WHERE compaction. Returns (dict of Columns, row ids)."""
        names = list(table.keys())
        cols = {k: self._dev(v) for k, v in table.items()}
        n = len(cols[names[0]])
        cap = n if out_cap is None else out_cap
        views = (_abi.ColView * len(names))(*[cols[k].view() for k in names])
        outs = {k: self._alloc(cols[k].dtype, cap, cols[k].validity is not None) for k in names}
        muts = (_abi.ColMut * len(names))(*[self._mut(outs[k], cap) for k in names])
        rid = torch.empty(max(cap, 1), dtype=torch.int32, device=f"cuda:{self.device}") if with_row_ids else None
        rmut = _abi.ColMut(rid.data_ptr(), None, cap, _abi.U32, 0) if with_row_ids else None
        n_out = C.c_uint64(0)
        if mask is not None:
            m = mask.to(f"cuda:{self.device}", dtype=torch.uint8)
            st = self._lib.bolt_compact_mask(self._ctx, views, len(names), C.c_void_p(m.data_ptr()), muts,
                                             C.byref(rmut) if rmut is not None else None, C.byref(n_out),
                                             flags | FLAG_PROFILE, C.c_void_p(self.stream_handle))
        else:
            preds = []
            for (cname, cmp, lit) in where:
                c = cols[cname]
                if c.dtype in ("f32", "f64"):
                    preds.append(_abi.Pred(names.index(cname), CMP_CODES[cmp], 0, float(lit)))
                else:
                    preds.append(_abi.Pred(names.index(cname), CMP_CODES[cmp], int(lit), 0.0))
            parr = (_abi.Pred * max(len(preds), 1))(*preds)
            st = self._lib.bolt_compact(self._ctx, views, len(names), parr, len(preds), muts,
                                        C.byref(rmut) if rmut is not None else None, C.byref(n_out),
                                        flags | FLAG_PROFILE, C.c_void_p(self.stream_handle))
        self._check(st, "compaction")
        k = int(n_out.value)
        res = {name: self._trim(outs[name], k) for name in names}
        return res, (rid[:k] if rid is not None else None)

    # ---- hash join ----------------------------------------------------------------
    def hash_join_indices(self, build_key: Column, probe_key: Column, out_cap: int | None = None,
                          flags: int = 0):
        """INNER equi-join: (probe_idx, build_idx) u32 pairs in probe order
        (hash_join_indices_on_gpu, src/exec/gpu_join.rs:1403); a build key
        that occurs several times pairs with each of its build rows in
        ascending row order (the reference's host join, src/exec/join.rs:
        407-425). Returns None on a decline (unsupported dtype). Without
        `out_cap` the output is sized to the probe rows and, when duplicate
        build keys produce more pairs, to the count the probe reports."""
        bk, pk = self._dev(build_key), self._dev(probe_key)
        table = C.c_void_p()
        st = self._lib.bolt_hash_join_build(self._ctx, C.byref(bk.view()), None, flags | FLAG_PROFILE,
                                            C.c_void_p(self.stream_handle), C.byref(table))
        if not self._check(st, "hash join build", decline_ok=True):
            return None
        try:
            cap = len(pk) if out_cap is None else out_cap
            for _attempt in range(2):
                pi = torch.empty(max(cap, 1), dtype=torch.int32, device=f"cuda:{self.device}")
                bi = torch.empty(max(cap, 1), dtype=torch.int32, device=f"cuda:{self.device}")
                n_out = C.c_uint64(0)
                st = self._lib.bolt_hash_join_probe(self._ctx, table, C.byref(pk.view()),
                                                    C.byref(_abi.ColMut(pi.data_ptr(), None, cap, _abi.U32, 0)),
                                                    C.byref(_abi.ColMut(bi.data_ptr(), None, cap, _abi.U32, 0)),
                                                    C.byref(n_out), flags | FLAG_PROFILE,
                                                    C.c_void_p(self.stream_handle))
                if st == _abi.ERR_CAPACITY and out_cap is None and int(n_out.value) > cap:
                    cap = int(n_out.value)
                    continue
                break
            self._check(st, "hash join probe")
            k = int(n_out.value)
            return pi[:k], bi[:k]
        finally:
            self._lib.bolt_hash_join_release(self._ctx, table)

    def join_groupby(self, build_key: Column, build_group: Column, probe_key: Column, value: Column,
                     max_groups: int = 1 << 16, flags: int = 0):
        """SELECT b.g, SUM(p.value), COUNT(*) FROM p JOIN b ON p.key = b.key
        GROUP BY b.g, without materialising the join. Returns
        (group Column, sum Column, count Column) sorted by group, or None on a
        decline (duplicate build keys: join with hash_join_indices instead)."""
        bk, bg, pk, val = self._dev(build_key), self._dev(build_group), self._dev(probe_key), self._dev(value)
        table = C.c_void_p()
        st = self._lib.bolt_hash_join_build(self._ctx, C.byref(bk.view()), C.byref(bg.view()),
                                            flags | FLAG_PROFILE, C.c_void_p(self.stream_handle), C.byref(table))
        if not self._check(st, "hash join build", decline_ok=True):
            return None
        try:
            sum_dt = _agg_out_dtype("sum", val.dtype)
            g = self._alloc("i32", max_groups, False)
            s = self._alloc(sum_dt, max_groups, False)
            s.scale = val.scale
            c = self._alloc("i64", max_groups, False)
            n_out = C.c_uint64(0)
            st = self._lib.bolt_join_groupby(self._ctx, table, C.byref(pk.view()), C.byref(val.view()),
                                             C.byref(self._mut(g, max_groups)), C.byref(self._mut(s, max_groups)),
                                             C.byref(self._mut(c, max_groups)), C.byref(n_out),
                                             flags | FLAG_PROFILE, C.c_void_p(self.stream_handle))
            if not self._check(st, "join GROUP BY", decline_ok=True):
                return None
            k = int(n_out.value)
            return self._trim(g, k), self._trim(s, k), self._trim(c, k)
        finally:
            self._lib.bolt_hash_join_release(self._ctx, table)


def _to_pinned_host(c: Column) -> Column:
    """Asynchronous device -> pinned host copy on the current stream (the
    caller synchronises once for all columns)."""
    def cp(t):
        h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
        h.copy_(t, non_blocking=True)
        return h
    return Column(cp(c.data), c.dtype, cp(c.validity) if c.validity is not None else None, c.scale)


class PreparedGroupby:
    """Descriptor + output columns of one GROUP BY through the C ABI. Keeps
    every buffer the descriptor points to alive."""

    def __init__(self, eng: Engine, cols: dict, group_by, aggs, where, groups_hint, out_cap, rows):
        self.eng = eng
        self.cols = cols
        names = list(cols.keys())
        self.views = (_abi.ColView * len(names))(*[cols[k].view() for k in names])
        self.key_idx = (C.c_int32 * len(group_by))(*[names.index(k) for k in group_by])
        preds = []
        for (cname, cmp, lit) in where:
            c = cols[cname]
            if c.dtype in ("f32", "f64"):
                preds.append(_abi.Pred(names.index(cname), CMP_CODES[cmp], 0, float(lit)))
            else:
                preds.append(_abi.Pred(names.index(cname), CMP_CODES[cmp], int(lit), 0.0))
        self.preds = (_abi.Pred * max(len(preds), 1))(*preds)
        specs, self.out_types, self.nullable, self.scales = [], [], [], []
        for (op, cname) in aggs:
            op = op.lower()
            if op == "count" and cname is None:
                op = "count_star"
            specs.append(_abi.AggSpec(AGG_CODES[op], names.index(cname) if cname is not None else -1))
            in_dt = cols[cname].dtype if cname is not None else None
            self.out_types.append(_agg_out_dtype(op, in_dt))
            self.nullable.append(cname is not None and cols[cname].validity is not None and op != "count")
            self.scales.append(cols[cname].scale if cname is not None else 0)
        self.specs = (_abi.AggSpec * len(specs))(*specs)
        self.group_by = group_by
        n = len(cols[group_by[0]])
        self.rows = rows if rows is not None else (0, n)
        span = self.rows[1] - self.rows[0]
        self.desc = _abi.GroupbyDesc(self.views, len(names), self.key_idx, len(group_by), self.preds, len(preds),
                                     self.specs, len(specs), groups_hint)
        self.realloc(out_cap if out_cap is not None else max(1, min(span + 1, max(2 * groups_hint, 1 << 16))))

    def realloc(self, cap: int):
        self.cap = cap
        e = self.eng
        key_null = len(self.group_by) == 1 and self.cols[self.group_by[0]].validity is not None
        self.kout = [e._alloc(self.cols[k].dtype, cap, key_null) for k in self.group_by]
        self.aout = [e._alloc(t, cap, nb) for t, nb in zip(self.out_types, self.nullable)]
        for c, sc in zip(self.aout, self.scales):
            if c.dtype == "dec128":
                c.scale = sc
        self.kmut = (_abi.ColMut * len(self.kout))(*[Engine._mut(c, cap) for c in self.kout])
        self.amut = (_abi.ColMut * len(self.aout))(*[Engine._mut(c, cap) for c in self.aout])
        self.out = _abi.GroupbyOut(self.kmut, self.amut, 0, None)

    def query(self) -> _abi.Query:
        return _abi.Query(self.desc, self.out, self.rows[0], self.rows[1], 0)

    def result(self, host_out: bool) -> GroupbyResult:
        g = int(self.out.n_groups)
        res = GroupbyResult([Engine._trim(c, g) for c in self.kout], [Engine._trim(c, g) for c in self.aout], g,
                            self.eng.last_device_ms, self.eng.last_launches)
        if host_out:
            res.keys = [_to_pinned_host(c) for c in res.keys]
            res.aggs = [_to_pinned_host(c) for c in res.aggs]
            torch.cuda.current_stream(self.eng.device).synchronize()
        return res


class BatchGraph:
    """A batch of prepared GROUP BY queries captured once as a CUDA graph
    (bolt_batch_graph_create) and replayed with one launch."""

    def __init__(self, device: int, prepared: Sequence[PreparedGroupby]):
        self._lib = lib()
        self.prepared = list(prepared)
        n = len(self.prepared)
        self.qs = (_abi.Query * n)(*[pq.query() for pq in self.prepared])
        h = C.c_void_p()
        st = self._lib.bolt_batch_graph_create(device, self.qs, n, C.byref(h))
        if st != _abi.OK:
            raise _ERRORS.get(st, BoltError)(f"bolt_batch_graph_create failed: {_abi.STATUS_NAMES[st]}", st)
        self._h = h
        self.device = device

    def launch(self, stream_handle: int | None = None):
        s = stream_handle if stream_handle is not None else torch.cuda.current_stream(self.device).cuda_stream
        st = self._lib.bolt_graph_launch(self._h, C.c_void_p(s))
        if st != _abi.OK:
            raise CudaError("bolt_graph_launch failed", st)

    def results(self, stream_handle: int | None = None) -> list[GroupbyResult]:
        s = stream_handle if stream_handle is not None else torch.cuda.current_stream(self.device).cuda_stream
        n = len(self.prepared)
        sts = (C.c_int32 * n)()
        ng = (C.c_uint64 * n)()
        st = self._lib.bolt_graph_sync_status(self._h, C.c_void_p(s), sts, ng)
        if st != _abi.OK:
            raise _ERRORS.get(st, BoltError)(f"batch graph replay: {_abi.STATUS_NAMES[st]}", st)
        out = []
        for i, pq in enumerate(self.prepared):
            pq.out.n_groups = ng[i]
            out.append(pq.result(False))
        return out

    def close(self):
        if getattr(self, "_h", None):
            self._lib.bolt_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching request loop (bolt_server_*): queries are admitted
    by HBM footprint into batches that run on `n_lanes` overlapping streams."""

    def __init__(self, device: int = 0, scratch_bytes: int = 0, max_batch: int = 256, n_lanes: int = 2):
        self._lib = lib()
        cfg = _abi.ServerConfig(device, scratch_bytes, max_batch, n_lanes)
        h = C.c_void_p()
        st = self._lib.bolt_server_create(C.byref(cfg), C.byref(h))
        if st != _abi.OK:
            raise _ERRORS.get(st, BoltError)(f"bolt_server_create failed: {_abi.STATUS_NAMES[st]}", st)
        self._h = h
        self._pending = {}

    def submit(self, pq: PreparedGroupby) -> int:
        q = _abi.Query(pq.desc, pq.out, pq.rows[0], pq.rows[1], 0)
        t = C.c_uint64(0)
        st = self._lib.bolt_server_submit(self._h, C.byref(q), C.byref(t))
        if st != _abi.OK:
            raise _ERRORS.get(st, BoltError)(f"bolt_server_submit failed: {_abi.STATUS_NAMES[st]}", st)
        self._pending[int(t.value)] = (pq, q)
        return int(t.value)

    def submit_many(self, pqs: Sequence[PreparedGroupby]) -> list[int]:
        """Submits a burst of queries in one call (bolt_server_submit_batch),
        so the lanes see it whole and form full batches."""
        n = len(pqs)
        qs = (_abi.Query * max(n, 1))(*[_abi.Query(pq.desc, pq.out, pq.rows[0], pq.rows[1], 0) for pq in pqs])
        ts = (C.c_uint64 * max(n, 1))()
        st = self._lib.bolt_server_submit_batch(self._h, qs, n, ts)
        if st != _abi.OK:
            raise _ERRORS.get(st, BoltError)(f"bolt_server_submit_batch failed: {_abi.STATUS_NAMES[st]}", st)
        out = []
        for i, pq in enumerate(pqs):
            t = int(ts[i])
            # The Query structs live in `qs`, which every pending entry keeps alive.
            self._pending[t] = (pq, qs[i], qs)
            out.append(t)
        return out

    def wait(self, ticket: int) -> tuple[GroupbyResult, float]:
        lat = C.c_double(0.0)
        st = self._lib.bolt_server_wait(self._h, ticket, C.byref(lat))
        pq, q = self._pending.pop(ticket)[:2]
        if st != _abi.OK:
            raise _ERRORS.get(st, BoltError)(f"query {ticket} failed: {_abi.STATUS_NAMES[st]}", st)
        pq.out.n_groups = q.out.n_groups
        return pq.result(False), float(lat.value)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.bolt_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
