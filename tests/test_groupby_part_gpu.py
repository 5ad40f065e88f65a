"""GPU parity: the hash-partitioned GROUP BY tier (groupby_part.cu) against
the oracle, and bit for bit against the shared-memory + global-hash-table
tier on the same input.

The partitioned tier serves dense inputs of 4M rows and more when the
caller forces it (FLAG_FORCE_PART, as here) or the autotuner found it the
faster tier for the query shape. Both tiers keep every
aggregate integer-exact (float64 sums as fixed point), so their outputs are
identical, not merely close. Covered here: the three key layouts it is
compiled for, with and without a WHERE conjunct, every compiled state
layout it serves, the key whose complement is zero, the retries after a
partition outgrows its table or the groups outgrow the group array, and
the hand-over to the global table for the row-order SUM(Int64) check.
"""

from __future__ import annotations

import importlib

import numpy as np
import pytest

from helpers import REL_TOL, compare_groupby

pytestmark = pytest.mark.gpu

N = 5_000_000  # the tier serves inputs of 4M rows and more


def tables(bolt, oracle, cols: dict):
    dev, host = {}, {}
    for name, (data, valid, dt, scale) in cols.items():
        dev[name] = bolt.col(data, dt, valid, scale).to("cuda")
        host[name] = oracle.HostCol(data, dt, valid, scale)
    return dev, host


def zipf_table(n: int, n_pairs: int, seed: int) -> dict:
    """(a, b) int32 halves of a mixed Zipf(1.1) rank, k64 int64 from the same
    mix, f int32 U[0,100), vd f64 N(0,1e3), vi int64 over most of the range,
    vs int64 |v| < 2^30, v32 int32."""
    dg = importlib.import_module("craton_bolt_b200.datagen")
    rng = np.random.default_rng(seed)
    r = np.minimum(rng.zipf(1.1, n), n_pairs).astype(np.uint64)
    h = dg.splitmix64(r ^ np.uint64(seed))
    a = (h >> np.uint64(32)).astype(np.uint32).view(np.int32)
    b = (h & np.uint64(0xFFFFFFFF)).astype(np.uint32).view(np.int32)
    return {"a": (a, None, "i32", 0), "b": (b, None, "i32", 0),
            "k64": ((h >> np.uint64(20)).view(np.int64), None, "i64", 0),
            "f": (rng.integers(0, 100, n).astype(np.int32), None, "i32", 0),
            "vd": (rng.normal(0, 1e3, n), None, "f64", 0),
            "vi": (rng.integers(-2**62, 2**62, n), None, "i64", 0),
            "vs": (rng.integers(-2**30, 2**30, n), None, "i64", 0),
            "v32": (rng.integers(-2**31, 2**31, n).astype(np.int32), None, "i32", 0)}


FILTERED_AGGS = [("sum", "vd"), ("avg", "vd"), ("count_star", None), ("min", "vi"), ("max", "vi")]


def run_tier(bolt, engine, oracle, cols, group_by, aggs, where=(), hint=0, want_tier=2, threads=8):
    """Runs the query forced onto the partitioned tier, checks which tier
    served it and compares with the oracle."""
    dev, host = tables(bolt, oracle, cols)
    res = engine.execute_groupby(dev, group_by, aggs, where=where, groups_hint=hint, flags=bolt.FLAG_FORCE_PART)
    assert engine.last_groupby_tier == want_tier
    orc = oracle.groupby(host, group_by, aggs, where=where, threads=threads)
    in_dts = [cols[c][2] if c is not None else None for _, c in aggs]
    compare_groupby(res, orc, [cols[k][2] for k in group_by], aggs, in_dts, REL_TOL)
    return res, dev


def same_bits(r1, r2):
    assert r1.n_groups == r2.n_groups
    for c1, c2 in zip(r1.keys + r1.aggs, r2.keys + r2.aggs):
        a, b = c1.numpy(), c2.numpy()
        assert np.array_equal(np.ascontiguousarray(a).view(np.uint8), np.ascontiguousarray(b).view(np.uint8))
        np.testing.assert_array_equal(c1.valid_mask(), c2.valid_mask())


def test_part_filtered_two_key_matches_oracle_and_global_tier(bolt, engine, oracle):
    """The benchmark's query shape: two int32 keys, WHERE f < 50, f64
    SUM/AVG, COUNT(*), int64 MIN/MAX."""
    cols = zipf_table(N, 2_000_000, 41)
    res, dev = run_tier(bolt, engine, oracle, cols, ["a", "b"], FILTERED_AGGS, [("f", "<", 50)], hint=600_000)
    assert res.n_groups > 200_000
    ref = engine.execute_groupby(dev, ["a", "b"], FILTERED_AGGS, where=[("f", "<", 50)], groups_hint=600_000,
                                 flags=bolt.FLAG_NO_PART)
    assert engine.last_groupby_tier == 1
    same_bits(res, ref)


@pytest.mark.parametrize("layout", ["i64_key_count_sum_max_min", "i32_key_where_sum_f64", "i64_key_count",
                                    "i32_key_sum_i32", "two_key_sum_i64"])
def test_part_compiled_layouts(bolt, engine, oracle, layout):
    cols = zipf_table(N, 1_000_000, 42)
    group_by, aggs, where = {
        "i64_key_count_sum_max_min": (["k64"], [("count_star", None), ("sum", "vs"), ("max", "vi"), ("min", "vd")], []),
        "i32_key_where_sum_f64": (["a"], [("sum", "vd"), ("count_star", None)], [("f", ">=", 30)]),
        "i64_key_count": (["k64"], [("count_star", None)], []),
        "i32_key_sum_i32": (["b"], [("sum", "v32"), ("count_star", None)], [("f", "!=", 7)]),
        "two_key_sum_i64": (["a", "b"], [("sum", "vs"), ("count_star", None)], []),
    }[layout]
    run_tier(bolt, engine, oracle, cols, group_by, aggs, where, hint=400_000)


def test_part_low_hint_retries(bolt, engine, oracle):
    """Forced onto the tier with a hint of 100 for ~400K groups: partitions
    outgrow their tables and the groups the array, and the retries still
    return the oracle's result on the partitioned tier."""
    cols = zipf_table(N, 1_000_000, 43)
    res, _ = run_tier(bolt, engine, oracle, cols, ["a", "b"], FILTERED_AGGS, [("f", "<", 80)], hint=100)
    assert res.n_groups > 100_000


def test_part_complement_zero_key(bolt, engine, oracle):
    """The key (-1, -1) packs to all ones, whose complement is the empty
    marker; it has its own slot and must come out as a normal group."""
    cols = zipf_table(N, 500_000, 44)
    a, b = cols["a"][0].copy(), cols["b"][0].copy()
    a[::97] = -1
    b[::97] = -1
    cols["a"] = (a, None, "i32", 0)
    cols["b"] = (b, None, "i32", 0)
    k64 = cols["k64"][0].copy()
    k64[::89] = -1
    cols["k64"] = (k64, None, "i64", 0)
    res, _ = run_tier(bolt, engine, oracle, cols, ["a", "b"], FILTERED_AGGS, [("f", "<", 50)], hint=300_000)
    keys = (res.keys[0].numpy().astype(np.int64), res.keys[1].numpy().astype(np.int64))
    assert ((keys[0] == -1) & (keys[1] == -1)).sum() == 1
    run_tier(bolt, engine, oracle, cols, ["k64"], [("count_star", None), ("sum", "vs")], hint=300_000)


def test_part_row_order_sum_check_uses_the_global_table(bolt, engine, oracle):
    """SUM(Int64) inputs of 2^50 over 5M rows could overflow in some row
    order, so the exact row-order check runs, which needs the global hash
    table: the query is served by tier 1 with the oracle's result."""
    cols = zipf_table(N, 1_000_000, 45)
    rng = np.random.default_rng(46)
    cols["vb"] = (rng.integers(-2**50, 2**50, N), None, "i64", 0)
    run_tier(bolt, engine, oracle, cols, ["a", "b"], [("sum", "vb"), ("count_star", None)], hint=400_000,
             want_tier=1)


def test_part_not_chosen_by_default(bolt, engine, oracle):
    """Untuned, the library serves the query with the global-table tier
    (the faster one on the measured shapes); the tuning cache or the flag
    selects the partitioned tier."""
    cols = zipf_table(N, 200_000, 48)
    dev, _ = tables(bolt, oracle, cols)
    engine.execute_groupby(dev, ["a", "b"], [("count_star", None)], groups_hint=400_000, flags=bolt.FLAG_NO_TUNE)
    assert engine.last_groupby_tier == 1


def test_part_everything_filtered(bolt, engine, oracle):
    cols = zipf_table(N, 100_000, 47)
    res, _ = run_tier(bolt, engine, oracle, cols, ["a", "b"], FILTERED_AGGS, [("f", "<", 0)], hint=100_000)
    assert res.n_groups == 0
