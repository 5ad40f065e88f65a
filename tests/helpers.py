"""Test helpers: golden fixtures, column conversion, result comparison."""

from __future__ import annotations

import json
import math
from pathlib import Path

import numpy as np

GOLDEN = Path(__file__).resolve().parent / "golden" / "known_answers.json"

# float64 SUM / AVG tolerance against the sequential FP64 oracle:
# |a - b| <= REL_TOL * max(|a|, |b|, 1)  (the reference's convention,
# tests/shmem_groupby_e2e.rs:150-160, tightened from its 1e-9 to 1e-12).
REL_TOL = 1e-12

NP_DT = {"i32": np.int32, "i64": np.int64, "f32": np.float32, "f64": np.float64, "u32": np.uint32}


def golden() -> dict:
    return json.loads(GOLDEN.read_text())


def _float(v):
    if isinstance(v, str):
        return {"NaN": math.nan, "inf": math.inf, "-inf": -math.inf}[v]
    return float(v)


def spec_arrays(spec: dict):
    """Golden column spec -> (numpy data, validity bitmap or None, dtype, scale)."""
    dt = spec["dtype"]
    vals = spec["values"]
    if dt == "dec128":
        ints = [int(v) for v in vals]
        lo = np.array([x & 0xFFFFFFFFFFFFFFFF for x in ints], dtype=np.uint64).view(np.int64)
        hi = np.array([(x >> 64) & 0xFFFFFFFFFFFFFFFF for x in ints], dtype=np.uint64).view(np.int64)
        data = np.stack([lo, hi], axis=1)
    elif dt in ("f32", "f64"):
        data = np.array([_float(v) for v in vals], dtype=NP_DT[dt])
    else:
        data = np.array(vals, dtype=NP_DT[dt])
    valid = None
    if "valid" in spec:
        valid = np.packbits(np.array(spec["valid"], dtype=np.uint8), bitorder="little")
    return data, valid, dt, spec.get("scale", 0)


def bitmap(mask: np.ndarray) -> np.ndarray:
    return np.packbits(mask.astype(np.uint8), bitorder="little")


def unpack_bits(bm, n: int) -> np.ndarray:
    if bm is None:
        return np.ones(n, dtype=bool)
    return np.unpackbits(np.asarray(bm, dtype=np.uint8), bitorder="little")[:n].astype(bool)


def split_packed(packed: np.ndarray, dtypes: list[str]) -> list[np.ndarray]:
    """Inverse of pack_keys for comparison: per key column raw values."""
    u = packed.astype(np.int64).view(np.uint64)
    if len(dtypes) == 1:
        dt = dtypes[0]
        if dt in ("i32", "f32"):
            return [(u & np.uint64(0xFFFFFFFF)).astype(np.uint32).view(np.int32 if dt == "i32" else np.float32)]
        return [u.view(np.int64 if dt == "i64" else np.float64)]
    a = (u >> np.uint64(32)).astype(np.uint32)
    b = (u & np.uint64(0xFFFFFFFF)).astype(np.uint32)
    return [a.view(np.int32 if dtypes[0] == "i32" else np.float32),
            b.view(np.int32 if dtypes[1] == "i32" else np.float32)]


def assert_float_close(got: np.ndarray, want: np.ndarray, rel: float = REL_TOL, what: str = "",
                       accurate: np.ndarray | None = None, stats: dict | None = None) -> int:
    """|got - want| <= rel * max(|got|, |want|, 1) against the sequential FP64
    oracle `want`. Where that fails, the value passes only if the oracle itself
    is the inaccurate one: `got` within rel of the compensated sum `accurate`
    while `want` is not (a group whose sum nearly cancels, or a group of
    millions of rows, can make a sequential fold's own rounding error exceed
    1e-12 * max(|S|, 1)). Returns how many values passed only that way (also
    added to stats[what] when `stats` is given)."""
    got = np.asarray(got, dtype=np.float64)
    want = np.asarray(want, dtype=np.float64)
    both_nan = np.isnan(got) & np.isnan(want)
    denom = np.maximum(np.maximum(np.abs(got), np.abs(want)), 1.0)
    with np.errstate(invalid="ignore"):
        bad = ~both_nan & ~(np.abs(got - want) <= rel * denom)
    escaped = 0
    if bad.any() and accurate is not None:
        acc = np.asarray(accurate, dtype=np.float64)
        d_acc = np.maximum(np.maximum(np.abs(got), np.abs(acc)), 1.0)
        with np.errstate(invalid="ignore"):
            got_ok = np.abs(got - acc) <= rel * d_acc
            oracle_off = ~(np.abs(want - acc) <= rel * d_acc)
        escaped = int((bad & got_ok & oracle_off).sum())
        bad = bad & ~(got_ok & oracle_off)
    if bad.any():
        i = int(np.flatnonzero(bad)[0])
        raise AssertionError(f"{what}: {int(bad.sum())} values differ, first at {i}: got {got[i]!r} want {want[i]!r}")
    if stats is not None:
        stats[what] = stats.get(what, 0) + escaped
    return escaped


def compare_groupby(res, orc: dict, group_by_dtypes: list[str], aggs: list, in_dtypes: list, rel: float = REL_TOL,
                    stats: dict | None = None):
    """Compares a GroupbyResult with the oracle's output (bit-exact except
    float SUM/AVG within `rel`; `stats` collects, per float aggregate, how many
    values passed through assert_float_close's compensated-sum check)."""
    g = orc["n_groups"]
    assert res.n_groups == g, f"group count {res.n_groups} != oracle {g}"
    want_keys = split_packed(orc["keys"], group_by_dtypes)
    for k, (kc, wk) in enumerate(zip(res.keys, want_keys)):
        got = kc.numpy()
        valid = unpack_bits(kc.validity.cpu().numpy() if kc.validity is not None else None, g)
        assert np.array_equal(~valid, orc["key_null"]), f"key {k} NULL flags differ"
        gv = got[valid].view(np.uint32 if got.dtype.itemsize == 4 else np.uint64)
        wv = wk[valid].view(np.uint32 if wk.dtype.itemsize == 4 else np.uint64)
        assert np.array_equal(gv, wv), f"key column {k} differs"
    for a, ((op, cname), in_dt) in enumerate(zip(aggs, in_dtypes)):
        ac = res.aggs[a]
        got = ac.numpy()
        want = orc["vals"][a]
        gvalid = unpack_bits(ac.validity.cpu().numpy() if ac.validity is not None else None, g)
        wvalid = orc["valid"][a]
        assert np.array_equal(gvalid, wvalid), f"aggregate {a} ({op}) NULL flags differ"
        m = wvalid
        if op in ("count", "count_star"):
            assert np.array_equal(got.astype(np.int64), want), f"aggregate {a} ({op}) differs"
        elif op == "sum" and in_dt == "dec128":
            assert np.array_equal(got[m], want[m]), f"aggregate {a} (SUM dec128) differs"
        elif op in ("avg",) or (op == "sum" and in_dt in ("f32", "f64")):
            acc = orc["accurate"][a][m] if in_dt in ("f32", "f64") else None
            assert_float_close(got[m], want[m], rel, f"aggregate {a} ({op})", accurate=acc, stats=stats)
        elif in_dt in ("f32", "f64"):
            gw = got[m].astype(np.float64)
            ww = want[m].astype(np.float64)
            same = (gw == ww) | (np.isnan(gw) & np.isnan(ww))
            assert same.all(), f"aggregate {a} ({op}) differs at {np.flatnonzero(~same)[:5]}"
        else:
            assert np.array_equal(got[m].astype(np.int64), want[m]), f"aggregate {a} ({op}) differs"
