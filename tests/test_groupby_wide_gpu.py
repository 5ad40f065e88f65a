"""GPU parity: GROUP BY over two integer key columns that do not pack into 64
bits (the sort-based wide-key path) against the oracle's restatement of the
reference's host wide reduction. Every result is a row-order fold, so the
comparison is bit-exact, floats included (NaN compared as NaN)."""

from __future__ import annotations

import numpy as np
import pytest

from helpers import bitmap, golden, spec_arrays

pytestmark = pytest.mark.gpu

AGGS = [("sum", "vi"), ("sum", "vd"), ("avg", "v32"), ("avg", "vi"), ("count_star", None), ("count", "vi"),
        ("min", "vd"), ("max", "vd"), ("min", "vf"), ("max", "vf"), ("min", "vi"), ("max", "v32")]


def _tables(bolt, oracle, cols):
    dev, host = {}, {}
    for name, (data, valid, dt) in cols.items():
        dev[name] = bolt.col(data, dt, valid).to("cuda")
        host[name] = oracle.HostCol(data, dt, valid)
    return dev, host


def _check(res, want, aggs):
    g = want["n_groups"]
    assert res.n_groups == g
    for k in range(2):
        assert np.array_equal(res.keys[k].numpy().astype(np.int64), want[f"k{k}"])
        assert res.keys[k].valid_mask().all()
    for i, (op, _c) in enumerate(aggs):
        col = res.aggs[i]
        assert np.array_equal(col.valid_mask(), want["valid"][i]), (op, _c)
        got, exp = col.numpy(), want["vals"][i]
        if got.dtype.kind == "f":
            got = got.astype(np.float64)
            nan = np.isnan(exp)
            assert np.array_equal(np.isnan(got), nan), (op, _c)
            assert np.array_equal(got[~nan].view(np.int64), exp[~nan].view(np.int64)), (op, _c)
        else:
            assert np.array_equal(got.astype(np.int64), exp), (op, _c)


def _columns(rng, n, kdt, distinct, key_nulls):
    k0 = rng.integers(-distinct, distinct + 1, n).astype(np.int64)
    k1 = rng.integers(-distinct, distinct + 1, n).astype(np.int64)
    if kdt[0] == "i64":
        k0 = k0 * (1 << 40) + 7
    if kdt[1] == "i64":
        k1 = k1 * -(1 << 33) - 3
    k0 = k0.astype(np.int32 if kdt[0] == "i32" else np.int64)
    k1 = k1.astype(np.int32 if kdt[1] == "i32" else np.int64)
    vi = rng.integers(-2 ** 62, 2 ** 62, n)  # sums wrap
    vd = rng.normal(0, 1e6, n)
    pick = rng.random(n)
    vd[pick < 0.05] = np.nan
    vd[(pick >= 0.05) & (pick < 0.10)] = -0.0
    vd[(pick >= 0.10) & (pick < 0.15)] = 0.0
    vf = rng.normal(0, 100, n).astype(np.float32)
    vf[rng.random(n) < 0.05] = np.nan
    v32 = rng.integers(-2 ** 31, 2 ** 31, n).astype(np.int32)
    vvalid = rng.random(n) > 0.3
    k0v = bitmap(rng.random(n) > 0.02) if key_nulls else None
    k1v = bitmap(rng.random(n) > 0.02) if key_nulls else None
    return {"k0": (k0, k0v, kdt[0]), "k1": (k1, k1v, kdt[1]), "vi": (vi, bitmap(vvalid), "i64"),
            "vd": (vd, bitmap(vvalid), "f64"), "vf": (vf, None, "f32"), "v32": (v32, None, "i32")}


@pytest.mark.parametrize("kdt", [("i64", "i64"), ("i64", "i32"), ("i32", "i64")])
@pytest.mark.parametrize("n,distinct", [(1, 1), (1000, 3), (300_000, 40), (300_000, 1 << 20)])
def test_groupby_wide_keys_match_oracle(bolt, engine, oracle, kdt, n, distinct):
    rng = np.random.default_rng(n + distinct + len(kdt[0]) * 7 + len(kdt[1]))
    cols = _columns(rng, n, kdt, distinct, key_nulls=True)
    dev, host = _tables(bolt, oracle, cols)
    res = engine.execute_groupby(dev, ["k0", "k1"], AGGS)
    assert engine.last_groupby_tier == 3
    _check(res, oracle.groupby_wide(host, ["k0", "k1"], AGGS), AGGS)


def test_groupby_wide_keys_without_nulls_and_large_groups(bolt, engine, oracle):
    """No key validity (no compaction before the sort) and three groups of
    about a million rows each (long row-order folds of one warp)."""
    rng = np.random.default_rng(5)
    cols = _columns(rng, 3_000_000, ("i64", "i32"), 1, key_nulls=False)
    cols["k1"] = (np.zeros(3_000_000, np.int32), None, "i32")
    dev, host = _tables(bolt, oracle, cols)
    res = engine.execute_groupby(dev, ["k0", "k1"], AGGS)
    assert res.n_groups == 3
    _check(res, oracle.groupby_wide(host, ["k0", "k1"], AGGS), AGGS)


def test_groupby_wide_keys_edge_cases(bolt, engine, oracle):
    rng = np.random.default_rng(9)
    cols = _columns(rng, 5000, ("i64", "i64"), 1 << 30, key_nulls=True)
    dev, host = _tables(bolt, oracle, cols)
    want = oracle.groupby_wide(host, ["k0", "k1"], AGGS)
    # Output capacity below the group count: ERR_CAPACITY, then the retry
    # with room for every group.
    _check(engine.execute_groupby(dev, ["k0", "k1"], AGGS, out_cap=3), want, AGGS)
    # Every key NULL: no groups.
    k = np.arange(64, dtype=np.int64)
    none = {"a": (k, bitmap(np.zeros(64, bool)), "i64"), "b": (k, None, "i64"), "v": (k, None, "i64")}
    d2, _ = _tables(bolt, oracle, none)
    assert engine.execute_groupby(d2, ["a", "b"], [("sum", "v"), ("count_star", None)]).n_groups == 0
    # The wide path is synchronous: an asynchronous call is declined.
    assert engine.try_execute_groupby(dev, ["k0", "k1"], AGGS, flags=bolt.FLAG_ASYNC) is None
    # SUM over Float32 has no wide-key form.
    assert engine.try_execute_groupby(dev, ["k0", "k1"], [("sum", "vf")]) is None


def test_groupby_wide_keys_host_columns(bolt, engine, oracle):
    """Host columns through bolt_groupby_host (the reference's RecordBatch
    entry): uploaded whole, then the same wide path; host results equal to the
    oracle."""
    rng = np.random.default_rng(17)
    cols = _columns(rng, 200_003, ("i32", "i64"), 300, key_nulls=True)
    host_cols = {name: bolt.col(d, dt, v) for name, (d, v, dt) in cols.items()}
    res = engine.execute_groupby(host_cols, ["k0", "k1"], AGGS)
    assert not res.keys[0].is_cuda and engine.last_groupby_tier == 3
    host = {name: oracle.HostCol(d, dt, v) for name, (d, v, dt) in cols.items()}
    _check(res, oracle.groupby_wide(host, ["k0", "k1"], AGGS), AGGS)


@pytest.mark.parametrize("case", golden()["groupby_wide"], ids=lambda c: c["name"])
def test_groupby_wide_known_answers(bolt, engine, case):
    """The reference's own wide GROUP BY tests (groupby_wide.rs) on the GPU."""
    dev = {}
    for name, spec in case["columns"].items():
        data, valid, dt, _ = spec_arrays(spec)
        dev[name] = bolt.col(data, dt, valid).to("cuda")
    exp = case["expected"]
    res = engine.execute_groupby(dev, case["group_by"], [tuple(a) for a in case["aggs"]])
    assert res.keys[0].numpy().tolist() == exp["k0"] and res.keys[1].numpy().tolist() == exp["k1"]
    for col, want in zip(res.aggs, exp["aggs"]):
        assert col.numpy().tolist() == want
