"""GPU parity: bolt_groupby (through the C ABI) against the CPU oracle."""

from __future__ import annotations

import math

import numpy as np
import pytest
import torch

from helpers import (REL_TOL, assert_float_close, bitmap, compare_groupby, golden, spec_arrays,
                     split_packed, unpack_bits)

pytestmark = pytest.mark.gpu


def tables(bolt, oracle, cols: dict):
    """numpy columns {name: (data, validity bitmap|None, dtype, scale)} ->
    (device Columns, oracle HostCols)."""
    dev, host = {}, {}
    for name, (data, valid, dt, scale) in cols.items():
        c = bolt.col(data, dt, valid, scale)
        dev[name] = c.to("cuda")
        host[name] = oracle.HostCol(data, dt, valid, scale)
    return dev, host


def run_both(bolt, engine, oracle, cols, group_by, aggs, where=(), hint=0, flags=0, rel=REL_TOL):
    dev, host = tables(bolt, oracle, cols)
    res = engine.execute_groupby(dev, group_by, aggs, where=where, groups_hint=hint, flags=flags)
    orc = oracle.groupby(host, group_by, aggs, where=where)
    in_dts = [cols[c][2] if c is not None else None for _, c in aggs]
    compare_groupby(res, orc, [cols[k][2] for k in group_by], aggs, in_dts, rel)
    return res, orc


@pytest.mark.parametrize("case", [c for c in golden()["groupby"] if "error" not in c["expected"]],
                         ids=lambda c: c["name"])
def test_groupby_known_answers(bolt, engine, oracle, case):
    cols = {k: spec_arrays(v) for k, v in case["columns"].items()}
    aggs = [tuple(a) for a in case["aggs"]]
    run_both(bolt, engine, oracle, cols, case["group_by"], aggs)


def test_groupby_decimal_overflow_known_answer(bolt, engine, oracle):
    case = [c for c in golden()["groupby"] if c["name"] == "decimal_sum_overflow"][0]
    cols = {k: spec_arrays(v) for k, v in case["columns"].items()}
    dev, _ = tables(bolt, oracle, cols)
    with pytest.raises(bolt.TypeError_) as ei:
        engine.execute_groupby(dev, ["k"], [("sum", "d")])
    assert "overflow" in str(ei.value) and "Decimal128" in str(ei.value)


def small_config(n, seed=1):
    import importlib
    dg = importlib.import_module("craton_bolt_b200.datagen")
    d = dg.groupby_small(n, seed)
    return {"k": (d["k"], None, "i32", 0), "v": (d["v"], None, "i64", 0)}


@pytest.mark.parametrize("flags_name", ["default", "force_global"])
def test_groupby_plain_single_key(bolt, engine, oracle, flags_name):
    """SELECT k, SUM(v), COUNT(*), MIN(v), MAX(v) GROUP BY k on 1,000,000 rows."""
    flags = bolt.FLAG_FORCE_GLOBAL if flags_name == "force_global" else 0
    cols = small_config(1_000_000)
    aggs = [("sum", "v"), ("count_star", None), ("min", "v"), ("max", "v")]
    res, orc = run_both(bolt, engine, oracle, cols, ["k"], aggs, hint=1024, flags=flags)
    assert res.n_groups == 1024


def test_groupby_plain_no_hint_grows(bolt, engine, oracle):
    cols = small_config(300_000, seed=5)
    aggs = [("sum", "v"), ("count_star", None)]
    run_both(bolt, engine, oracle, cols, ["k"], aggs, hint=0)


def filtered_config(n, n_pairs, seed=2):
    import importlib
    dg = importlib.import_module("craton_bolt_b200.datagen")
    d = dg.groupby_filtered(n, seed, n_pairs=n_pairs)
    return {"a": (d["a"], None, "i32", 0), "b": (d["b"], None, "i32", 0), "f": (d["f"], None, "i32", 0),
            "vd": (d["vd"], None, "f64", 0), "vi": (d["vi"], None, "i64", 0)}


FILTERED_AGGS = [("sum", "vd"), ("avg", "vd"), ("count_star", None), ("min", "vi"), ("max", "vi")]


@pytest.mark.parametrize("n,n_pairs,hint", [(200_000, 50_000, 0), (2_000_000, 1_000_000, 400_000),
                                            (3_000_000, 10_000_000, 0)])
def test_groupby_filtered_two_key(bolt, engine, oracle, n, n_pairs, hint):
    """Filtered high-cardinality two-key GROUP BY (Zipf pairs, f < 50)."""
    cols = filtered_config(n, n_pairs)
    res, orc = run_both(bolt, engine, oracle, cols, ["a", "b"], FILTERED_AGGS, where=[("f", "<", 50)], hint=hint)
    assert res.n_groups > 1000


KERNELS = ["regs", "staged"]


def kernel_flags(bolt, kernel):
    return bolt.FLAG_KERNEL_STAGED if kernel == "staged" else bolt.FLAG_KERNEL_REGS


@pytest.mark.parametrize("kernel", KERNELS)
def test_groupby_filtered_two_key_kernels(bolt, engine, oracle, kernel):
    """Both aggregation kernels on the filtered two-key shape; the row count is
    not a multiple of any tile, so the staged kernel also folds a remainder."""
    cols = filtered_config(2_000_077, 1_000_000, seed=17)
    res, _ = run_both(bolt, engine, oracle, cols, ["a", "b"], FILTERED_AGGS, where=[("f", "<", 50)],
                      hint=400_000, flags=kernel_flags(bolt, kernel))
    assert res.n_groups > 1000


def test_groupby_staged_matches_register_kernel_bitwise(bolt, engine, oracle):
    cols = filtered_config(1_000_003, 50_000, seed=21)
    dev, _ = tables(bolt, oracle, cols)
    r1 = engine.execute_groupby(dev, ["a", "b"], FILTERED_AGGS, where=[("f", "<", 50)],
                                flags=bolt.FLAG_KERNEL_REGS)
    r2 = engine.execute_groupby(dev, ["a", "b"], FILTERED_AGGS, where=[("f", "<", 50)],
                                flags=bolt.FLAG_KERNEL_STAGED)
    assert r1.n_groups == r2.n_groups
    for x, y in zip(r1.keys + r1.aggs, r2.keys + r2.aggs):
        xd = x.data.view(torch.int64) if x.dtype == "f64" else x.data
        yd = y.data.view(torch.int64) if y.dtype == "f64" else y.data
        assert torch.equal(xd, yd)


@pytest.mark.parametrize("kernel", KERNELS)
@pytest.mark.parametrize("layout", ["count_sum_i64", "count", "count_sum_i32", "count_sum_f64"])
def test_groupby_compiled_layouts(bolt, engine, oracle, kernel, layout):
    """Each compiled state layout, with NULL single keys, f32 / i32 keys and
    WHERE conjuncts over i32, i64 and f64 columns."""
    rng = np.random.default_rng(23)
    n = 700_001
    k = rng.integers(-3000, 3000, n).astype(np.int32)
    kv = rng.random(n) > 0.01
    kf = (rng.integers(-400, 400, n) / 8.0).astype(np.float32)
    x = rng.normal(0, 1, n)
    y = rng.integers(-2**40, 2**40, n).astype(np.int64)
    z = rng.integers(-2**30, 2**30, n).astype(np.int32)
    f = rng.integers(0, 100, n).astype(np.int32)
    cols = {"k": (k, bitmap(kv), "i32", 0), "kf": (kf, None, "f32", 0), "x": (x, None, "f64", 0),
            "y": (y, None, "i64", 0), "z": (z, None, "i32", 0), "f": (f, None, "i32", 0)}
    where = [("f", "<", 70), ("x", ">", -1.5), ("y", "!=", 12345)]
    aggs = {"count_sum_i64": [("sum", "y"), ("count_star", None)],
            "count": [("count_star", None)],
            "count_sum_i32": [("count_star", None), ("sum", "z")],
            "count_sum_f64": [("avg", "x")]}[layout]
    flags = kernel_flags(bolt, kernel)
    run_both(bolt, engine, oracle, cols, ["k"], aggs, where=where, flags=flags)
    run_both(bolt, engine, oracle, cols, ["kf"], aggs, where=where[:1], flags=flags)


def test_groupby_staged_unaligned_columns_fall_back(bolt, engine, oracle):
    """Columns that start off a 16-byte boundary take the register kernel."""
    d = small_config(500_001, seed=29)
    k = torch.from_numpy(d["k"][0]).to("cuda")
    v = torch.from_numpy(d["v"][0]).to("cuda")
    dev = {"k": bolt.Column(k[1:], "i32"), "v": bolt.Column(v[1:], "i64")}
    host = {"k": oracle.HostCol(d["k"][0][1:].copy(), "i32"), "v": oracle.HostCol(d["v"][0][1:].copy(), "i64")}
    aggs = [("sum", "v"), ("count_star", None)]
    res = engine.execute_groupby(dev, ["k"], aggs, groups_hint=1024, flags=bolt.FLAG_KERNEL_STAGED)
    compare_groupby(res, oracle.groupby(host, ["k"], aggs), ["i32"], aggs, ["i64", None], REL_TOL)


def test_groupby_f64_sum_is_order_independent(bolt, engine, oracle):
    """Fixed-point f64 sums: bit-identical across runs and table tiers."""
    cols = filtered_config(500_000, 20_000, seed=7)
    dev, _ = tables(bolt, oracle, cols)
    r1 = engine.execute_groupby(dev, ["a", "b"], FILTERED_AGGS, where=[("f", "<", 50)])
    r2 = engine.execute_groupby(dev, ["a", "b"], FILTERED_AGGS, where=[("f", "<", 50)], flags=bolt.FLAG_FORCE_GLOBAL)
    for x, y in zip(r1.aggs, r2.aggs):
        assert torch.equal(x.data.view(torch.int64) if x.dtype == "f64" else x.data,
                           y.data.view(torch.int64) if y.dtype == "f64" else y.data)


def test_groupby_f64_sum_close_to_exact(bolt, engine, oracle):
    """The fixed-point SUM is within one ulp of the compensated (accurate) sum."""
    cols = filtered_config(400_000, 5_000, seed=11)
    dev, host = tables(bolt, oracle, cols)
    res = engine.execute_groupby(dev, ["a", "b"], [("sum", "vd")], where=[("f", "<", 50)])
    orc = oracle.groupby(host, ["a", "b"], [("sum", "vd")], where=[("f", "<", 50)])
    got = res.aggs[0].numpy()
    acc = orc["accurate"][0]
    ulp = np.spacing(np.abs(acc))
    assert np.all(np.abs(got - acc) <= ulp + 1e-15)


@pytest.mark.parametrize("tier", ["default", "force_global"])
@pytest.mark.parametrize("with_out_of_window", [False, True])
def test_groupby_f64_sum_window_edges(bolt, engine, oracle, tier, with_out_of_window):
    """f64 SUM / AVG at the edges of the fixed-point window: magnitudes just
    below 2^32 (the global table's signed high word then carries its largest
    sums), tiny and subnormal values, signed zeros and cancelling signs, in
    both tiers. With a value of magnitude 2^32 the call falls back to f64
    atomics and still meets the tolerance."""
    rng = np.random.default_rng(31)
    n = 200_000
    pool = np.array([4294967295.5, -4294967295.5, 4294967296.0 - 2.0 ** -20, -(4294967296.0 - 2.0 ** -20),
                     1e-300, -1e-300, 5e-324, 0.0, -0.0, 1.0, -1.0, 123456.789], dtype=np.float64)
    v = pool[rng.integers(0, len(pool), n)]
    if with_out_of_window:
        # The fallback's f64 atomics round in arrival order: non-negative
        # values keep every partial sum below the final one, so its rounding
        # error stays within the tolerance whatever the order.
        v = np.abs(v)
        v[::997] = 4294967296.0
    k = rng.integers(0, 64, n).astype(np.int32)
    cols = {"k": (k, None, "i32", 0), "v": (v, None, "f64", 0)}
    aggs = [("sum", "v"), ("avg", "v"), ("count_star", None)]
    flags = bolt.FLAG_FORCE_GLOBAL if tier == "force_global" else 0
    run_both(bolt, engine, oracle, cols, ["k"], aggs, hint=64, flags=flags)


def test_groupby_null_keys_and_values(bolt, engine, oracle):
    rng = np.random.default_rng(3)
    n = 100_000
    k = rng.integers(-500, 500, n).astype(np.int32)
    kv = rng.random(n) > 0.02
    v = rng.integers(-2**40, 2**40, n).astype(np.int64)
    vv = rng.random(n) > 0.3
    d = rng.normal(0, 5, n)
    dv = rng.random(n) > 0.5
    cols = {"k": (k, bitmap(kv), "i32", 0), "v": (v, bitmap(vv), "i64", 0), "d": (d, bitmap(dv), "f64", 0)}
    aggs = [("count_star", None), ("count", "v"), ("sum", "v"), ("min", "v"), ("max", "v"), ("avg", "d"),
            ("min", "d")]
    run_both(bolt, engine, oracle, cols, ["k"], aggs)


def test_groupby_key_dtypes(bolt, engine, oracle):
    rng = np.random.default_rng(4)
    n = 50_000
    base = rng.integers(0, 300, n)
    cases = {
        "i64": (base.astype(np.int64) * 1_000_000_007 - 2**62, "i64"),
        "f64": (np.where(base % 7 == 0, -0.0, base / 3.0 - 20.0), "f64"),
        "f32": (np.where(base % 5 == 0, np.float32(np.nan), (base / 7.0).astype(np.float32)).astype(np.float32), "f32"),
    }
    for name, (kd, dt) in cases.items():
        cols = {"k": (kd, None, dt, 0), "v": (base.astype(np.int32), None, "i32", 0)}
        run_both(bolt, engine, oracle, cols, ["k"], [("sum", "v"), ("count_star", None), ("max", "v")])


def test_groupby_sentinel_key_minus_one(bolt, engine, oracle):
    """Key -1 packs to all ones (the value whose complement marks empty slots)."""
    k = np.array([-1, 5, -1, 7, -1, 5], np.int32)
    v = np.arange(6, dtype=np.int64)
    run_both(bolt, engine, oracle, {"k": (k, None, "i32", 0), "v": (v, None, "i64", 0)}, ["k"],
             [("sum", "v"), ("count_star", None)])
    a = np.array([-1, -1, 0, -1], np.int32)
    b = np.array([-1, -1, 0, 3], np.int32)
    run_both(bolt, engine, oracle, {"a": (a, None, "i32", 0), "b": (b, None, "i32", 0)}, ["a", "b"],
             [("count_star", None)])


def test_groupby_sum_i64_overflow(bolt, engine, oracle):
    k = np.zeros(4, np.int32)
    v = np.array([2**62, 2**62, 5, 7], np.int64)
    dev, _ = tables(bolt, oracle, {"k": (k, None, "i32", 0), "v": (v, None, "i64", 0)})
    with pytest.raises(bolt.TypeError_) as ei:
        engine.execute_groupby(dev, ["k"], [("sum", "v")])
    assert "SUM(integer) overflow" in str(ei.value)


@pytest.mark.parametrize("order,overflows", [((1, 1, -1, -1), True), ((1, -1, 1, -1), False)])
def test_groupby_sum_i64_row_order_prefix_overflow(bolt, engine, oracle, order, overflows):
    """checked_group_sum errors when a row-order prefix leaves i64 even if the
    final sum fits; the GPU path reproduces that exactly."""
    k = np.array([0, 1, 0, 1, 0, 1, 0, 1], np.int32)
    v = np.array([s * 2**62 for s in order for _ in range(2)], np.int64)
    dev, host = tables(bolt, oracle, {"k": (k, None, "i32", 0), "v": (v, None, "i64", 0)})
    if overflows:
        with pytest.raises(bolt.TypeError_):
            engine.execute_groupby(dev, ["k"], [("sum", "v")])
        with pytest.raises(oracle.OracleError):
            oracle.groupby(host, ["k"], [("sum", "v")])
    else:
        res = engine.execute_groupby(dev, ["k"], [("sum", "v")])
        assert res.aggs[0].numpy().tolist() == [0, 0]
        assert oracle.groupby(host, ["k"], [("sum", "v")])["vals"][0].tolist() == [0, 0]


def test_groupby_empty_input_and_all_filtered(bolt, engine, oracle):
    k = np.zeros(0, np.int32)
    v = np.zeros(0, np.int64)
    res, _ = run_both(bolt, engine, oracle, {"k": (k, None, "i32", 0), "v": (v, None, "i64", 0)}, ["k"],
                      [("sum", "v")])
    assert res.n_groups == 0
    k = np.arange(1000, dtype=np.int32)
    f = np.full(1000, 99, np.int32)
    res, _ = run_both(bolt, engine, oracle, {"k": (k, None, "i32", 0), "f": (f, None, "i32", 0)}, ["k"],
                      [("count_star", None)], where=[("f", "<", 50)])
    assert res.n_groups == 0


def test_groupby_single_hot_key(bolt, engine, oracle):
    """Every row in one group (maximal atomic contention)."""
    n = 2_000_000
    k = np.full(n, 42, np.int32)
    v = np.random.default_rng(8).integers(-1000, 1000, n).astype(np.int64)
    d = np.random.default_rng(9).normal(0, 1e3, n)
    run_both(bolt, engine, oracle, {"k": (k, None, "i32", 0), "v": (v, None, "i64", 0), "d": (d, None, "f64", 0)},
             ["k"], [("sum", "v"), ("sum", "d"), ("count_star", None), ("min", "v"), ("max", "d")])


def test_groupby_nonfinite_f64_falls_back(bolt, engine, oracle):
    k = np.array([0, 0, 1, 1, 2, 2], np.int32)
    d = np.array([1.0, np.inf, 2.0, 3.0, 1e300, 1e300], np.float64)
    dev, host = tables(bolt, oracle, {"k": (k, None, "i32", 0), "d": (d, None, "f64", 0)})
    res = engine.execute_groupby(dev, ["k"], [("sum", "d")])
    got = res.aggs[0].numpy()
    assert got[0] == np.inf and got[1] == 5.0 and got[2] == 2e300


def test_groupby_where_float_and_multiple_conjuncts(bolt, engine, oracle):
    rng = np.random.default_rng(12)
    n = 200_000
    cols = {"k": (rng.integers(0, 2000, n).astype(np.int32), None, "i32", 0),
            "x": (rng.normal(0, 1, n), None, "f64", 0),
            "y": (rng.integers(-100, 100, n).astype(np.int64), None, "i64", 0)}
    run_both(bolt, engine, oracle, cols, ["k"], [("sum", "y"), ("avg", "x"), ("count_star", None)],
             where=[("x", ">", 0.25), ("y", "!=", 3), ("y", ">=", -50)])


def test_groupby_decline_unsupported(bolt, engine, oracle):
    k = np.zeros(4, np.float64)
    v = np.zeros(4, np.int64)
    dev, _ = tables(bolt, oracle, {"a": (k, None, "f64", 0), "b": (v, None, "i64", 0)})
    assert engine.try_execute_groupby(dev, ["a", "b"], [("count_star", None)]) is None


def test_groupby_host_inputs_end_to_end(bolt, engine, oracle):
    """Host numpy columns in, host columns out (the end-to-end path)."""
    cols = small_config(100_000, seed=9)
    host = {k: bolt.col(v[0], v[2]) for k, v in cols.items()}
    res = engine.execute_groupby(host, ["k"], [("sum", "v"), ("count_star", None)], groups_hint=1024)
    assert not res.keys[0].is_cuda
    orc = oracle.groupby({k: oracle.HostCol(v[0], v[2]) for k, v in cols.items()}, ["k"],
                         [("sum", "v"), ("count_star", None)])
    compare_groupby(res, orc, ["i32"], [("sum", "v"), ("count_star", None)], ["i64", None])


def test_groupby_host_columns_streamed_in_chunks(bolt, engine, oracle):
    """Host columns through bolt_groupby_host: more rows than one 4M-row
    chunk (plus a remainder), a nullable single key, nullable values and a
    WHERE; equal to the oracle and bit-identical to the device-column path."""
    rng = np.random.default_rng(41)
    n = 9_000_013
    k = rng.integers(-20000, 20000, n).astype(np.int32)
    kv = rng.random(n) > 0.001
    v = rng.integers(-10**9, 10**9, n).astype(np.int64)
    vv = rng.random(n) > 0.05
    d = rng.normal(0, 100, n)
    f = rng.integers(0, 100, n).astype(np.int32)
    cols = {"k": (k, bitmap(kv), "i32", 0), "v": (v, bitmap(vv), "i64", 0), "d": (d, None, "f64", 0),
            "f": (f, None, "i32", 0)}
    aggs = [("sum", "v"), ("count", "v"), ("avg", "d"), ("max", "d"), ("count_star", None)]
    where = [("f", ">=", 20)]
    host = {name: bolt.Column(torch.from_numpy(a).pin_memory(), dt,
                              torch.from_numpy(vb).pin_memory() if vb is not None else None, sc)
            for name, (a, vb, dt, sc) in cols.items()}
    res = engine.execute_groupby(host, ["k"], aggs, where=where, groups_hint=40_000)
    assert not res.keys[0].is_cuda
    hcols = {name: oracle.HostCol(a, dt, vb, sc) for name, (a, vb, dt, sc) in cols.items()}
    orc = oracle.groupby(hcols, ["k"], aggs, where=where)
    compare_groupby(res, orc, ["i32"], aggs, ["i64", "i64", "f64", "f64", None])
    dev, _ = tables(bolt, oracle, cols)
    r2 = engine.execute_groupby(dev, ["k"], aggs, where=where, groups_hint=40_000)
    assert r2.n_groups == res.n_groups
    for x, y in zip(res.keys + res.aggs, r2.keys + r2.aggs):
        np.testing.assert_array_equal(x.valid_mask(), y.valid_mask())
        xd, yd = x.numpy(), y.numpy()
        if x.dtype == "f64":
            xd, yd = xd.view(np.int64), yd.view(np.int64)
        np.testing.assert_array_equal(xd[x.valid_mask()], yd[y.valid_mask()])


def test_groupby_host_columns_row_order_check_falls_back(bolt, engine, oracle):
    """A SUM(Int64) that needs the row-order overflow check is declined by the
    streamed path and run on device columns instead: same error as bolt_groupby."""
    k = np.array([0, 1, 0, 1, 0, 1, 0, 1], np.int32)
    v = np.array([s * 2**62 for s in (1, 1, -1, -1) for _ in range(2)], np.int64)
    host = {"k": bolt.col(k, "i32"), "v": bolt.col(v, "i64")}
    with pytest.raises(bolt.TypeError_):
        engine.execute_groupby(host, ["k"], [("sum", "v")])
    v2 = np.array([s * 2**62 for s in (1, -1, 1, -1) for _ in range(2)], np.int64)
    res = engine.execute_groupby({"k": bolt.col(k, "i32"), "v": bolt.col(v2, "i64")}, ["k"], [("sum", "v")])
    assert res.aggs[0].numpy().tolist() == [0, 0]


def test_autotune_keeps_results_and_persists(bolt, engine, oracle, tmp_path):
    cols = filtered_config(1_000_000, 100_000, seed=13)
    dev, host = tables(bolt, oracle, cols)
    base = engine.execute_groupby(dev, ["a", "b"], FILTERED_AGGS, where=[("f", "<", 50)], groups_hint=100_000,
                                  flags=bolt.FLAG_NO_TUNE)
    pq = engine.prepare_groupby(dev, ["a", "b"], FILTERED_AGGS, [("f", "<", 50)], groups_hint=100_000)
    best = engine.autotune_groupby(pq)
    assert best > 0
    tuned = engine.execute_groupby(dev, ["a", "b"], FILTERED_AGGS, where=[("f", "<", 50)], groups_hint=100_000)
    for x, y in zip(base.aggs + base.keys, tuned.aggs + tuned.keys):
        xa = x.data.view(torch.int64) if x.data.dtype == torch.float64 else x.data
        ya = y.data.view(torch.int64) if y.data.dtype == torch.float64 else y.data
        assert torch.equal(xa, ya)
    path = tmp_path / "tune.txt"
    engine.save_tuning(path)
    assert path.read_text().strip()
    other = bolt.Engine(0, scratch_bytes=1 << 30)
    try:
        other.load_tuning(path)
    finally:
        other.close()
