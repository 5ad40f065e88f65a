"""CPU: the oracle against the reference's known answers and an independent
pure-Python restatement on small seeded inputs."""

from __future__ import annotations

import math

import numpy as np
import pytest

from helpers import golden, spec_arrays, split_packed, unpack_bits


def host_table(oracle, columns: dict) -> dict:
    out = {}
    for name, spec in columns.items():
        data, valid, dt, scale = spec_arrays(spec)
        out[name] = oracle.HostCol(data, dt, valid, scale)
    return out


def _eq(a, b) -> bool:
    if isinstance(b, float) or isinstance(a, float):
        a, b = float(a), float(b)
        return (math.isnan(a) and math.isnan(b)) or a == b
    return int(a) == int(b)


@pytest.mark.parametrize("case", golden()["groupby"], ids=lambda c: c["name"])
def test_oracle_groupby_known_answers(oracle, case):
    t = host_table(oracle, case["columns"])
    exp = case["expected"]
    aggs = [tuple(a) for a in case["aggs"]]
    if "error" in exp:
        with pytest.raises(oracle.OracleError) as ei:
            oracle.groupby(t, case["group_by"], aggs)
        assert ei.value.status == oracle.OVERFLOW
        for word in exp["message_contains"]:
            assert word in str(ei.value)
        return
    r = oracle.groupby(t, case["group_by"], aggs)
    assert r["n_groups"] == len(exp["keys"])
    dts = [case["columns"][k]["dtype"] for k in case["group_by"]]
    keys = split_packed(r["keys"], dts)
    for g, want in enumerate(exp["keys"]):
        if want == [None]:
            assert r["key_null"][g]
            continue
        assert not r["key_null"][g]
        assert [int(k[g]) for k in keys] == want
    for a, (vals, valid) in enumerate(zip(exp["aggs"], exp["agg_valid"])):
        for g in range(len(vals)):
            assert bool(r["valid"][a][g]) == bool(valid[g]), (case["name"], a, g)
            if not valid[g]:
                continue
            got = r["vals"][a][g]
            if case["columns"].get(aggs[a][1] or "", {}).get("dtype") == "dec128":
                lo, hi = int(got[0]) & (2**64 - 1), int(got[1])
                got = (hi << 64) | lo
            want = vals[g]
            if want == "NaN":
                want = math.nan
            assert _eq(got, want), (case["name"], a, g, got, want)


@pytest.mark.parametrize("case", golden()["join"], ids=lambda c: c["name"])
def test_oracle_join_known_answers(oracle, case):
    bd, bv, bdt, _ = spec_arrays(case["build"])
    pd, pv, pdt, _ = spec_arrays(case["probe"])
    b = oracle.HostCol(bd, bdt, bv)
    p = oracle.HostCol(pd, pdt, pv)
    pr, br = oracle.hash_join(b, p)
    assert len(pr) == case["expected"]["n_pairs"]
    if len(pr):
        pk = spec_arrays(case["probe"])[0]
        bk = spec_arrays(case["build"])[0]
        assert np.array_equal(bk[br], pk[pr])
        assert np.all(np.diff(pr.astype(np.int64)) > 0)  # probe order


@pytest.mark.parametrize("case", golden()["sort_keys"], ids=lambda c: c["name"])
def test_oracle_sort_key_transform(oracle, case):
    dt = case["dtype"]
    if "bits" in case:
        data = np.array(case["bits"], dtype=np.uint32).view(np.float32)
    else:
        data = np.array([float(v) for v in case["values"]], dtype=np.float32 if dt == "f32" else np.float64)
    k = oracle.sort_keys(oracle.HostCol(data, dt), case.get("descending", False)).astype(np.uint64)
    prop = case["property"]
    if prop == "strictly_increasing":
        assert np.all(np.diff(k.astype(object)) > 0)
    elif prop == "strictly_decreasing":
        assert np.all(np.diff(k.astype(object)) < 0)
    elif prop == "all_equal":
        assert len(set(k.tolist())) == 1
    else:
        assert len(set(k.tolist())) == 1
        inf = oracle.sort_keys(oracle.HostCol(np.array([np.inf], np.float32), "f32"))[0]
        assert int(k[0]) > int(inf)


def sort_input(oracle, case):
    n = case["n"]
    if case["gen"] == "shuffle_iota":
        v = oracle.shuffle_deterministic(np.arange(n, dtype=np.uint32), case["seed"]).view(np.int32)
        return v.astype(np.int32)
    if case["gen"] == "mul7919_mod_shuffle":
        base = (np.arange(n, dtype=np.int64) * 7919) % 1_000_000
        idx = oracle.shuffle_deterministic(np.arange(n, dtype=np.uint32), case["seed"]).astype(np.int64)
        return base[idx]
    return np.sin(np.arange(n, dtype=np.float64) * 1.61803398875)


@pytest.mark.parametrize("case", golden()["sort"], ids=lambda c: c["name"])
def test_oracle_sort_known_answers(oracle, case):
    v = sort_input(oracle, case)
    perm = oracle.sort_perm(oracle.HostCol(v, case["dtype"]), case["descending"])
    out = v[perm]
    want = np.sort(v)[::-1] if case["descending"] else np.sort(v)
    assert np.array_equal(out, want)
    # stability: equal keys keep input order
    same = out[1:] == out[:-1]
    assert np.all(perm[1:][same] > perm[:-1][same])


def test_shuffle_deterministic_is_a_permutation(oracle):
    a = oracle.shuffle_deterministic(np.arange(1000, dtype=np.uint32), 7)
    assert sorted(a.tolist()) == list(range(1000))
    assert not np.array_equal(a, np.arange(1000))


def test_xorshift64star_matches_python_restatement(oracle):
    seed = 0xB2
    s = (seed + 0x9E3779B97F4A7C15) & (2**64 - 1)
    want = []
    for _ in range(64):
        s ^= s >> 12
        s ^= (s << 25) & (2**64 - 1)
        s ^= s >> 27
        want.append((s * 0x2545F4914F6CDD1D) & (2**64 - 1))
    assert oracle.xorshift64star(seed, 64).tolist() == want


# ---------------------------------------------------------------------------
# Independent pure-Python restatement (small sizes only)
# ---------------------------------------------------------------------------
def py_groupby(k, kvalid, v, vvalid, f, lit):
    groups = {}
    for i in range(len(k)):
        if not (f[i] < lit):
            continue
        key = None if not kvalid[i] else int(k[i])
        g = groups.setdefault(key, {"cnt": 0, "n": 0, "sum": 0, "min": None, "max": None, "fsum": 0.0})
        g["cnt"] += 1
        if vvalid[i]:
            x = int(v[i])
            g["n"] += 1
            g["sum"] += x
            g["fsum"] += float(x)
            g["min"] = x if g["min"] is None else min(g["min"], x)
            g["max"] = x if g["max"] is None else max(g["max"], x)
    order = sorted([kk for kk in groups if kk is not None]) + ([None] if None in groups else [])
    return order, groups


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_groupby_matches_python(oracle, seed):
    rng = np.random.default_rng(seed)
    n = 3000
    k = rng.integers(-50, 50, n).astype(np.int32)
    kvalid = rng.random(n) > 0.05
    v = rng.integers(-10**6, 10**6, n).astype(np.int64)
    vvalid = rng.random(n) > 0.1
    f = rng.integers(0, 100, n).astype(np.int32)
    bm = lambda m: np.packbits(m.astype(np.uint8), bitorder="little")
    t = {"k": oracle.HostCol(k, "i32", bm(kvalid)), "v": oracle.HostCol(v, "i64", bm(vvalid)),
         "f": oracle.HostCol(f, "i32")}
    aggs = [("count_star", None), ("count", "v"), ("sum", "v"), ("min", "v"), ("max", "v"), ("avg", "v")]
    r = oracle.groupby(t, ["k"], aggs, where=[("f", "<", 50)])
    order, groups = py_groupby(k, kvalid, v, vvalid, f, 50)
    assert r["n_groups"] == len(order)
    for gi, key in enumerate(order):
        g = groups[key]
        assert r["key_null"][gi] == (key is None)
        if key is not None:
            assert int(r["keys"][gi]) == key
        assert r["vals"][0][gi] == g["cnt"]
        assert r["vals"][1][gi] == g["n"]
        assert bool(r["valid"][2][gi]) == (g["n"] > 0)
        if g["n"]:
            assert r["vals"][2][gi] == g["sum"]
            assert r["vals"][3][gi] == g["min"]
            assert r["vals"][4][gi] == g["max"]
            assert r["vals"][5][gi] == g["fsum"] / g["n"]


def test_oracle_two_key_packing_and_order(oracle):
    a = np.array([1, -1, 1, 0, -1], np.int32)
    b = np.array([-1, 5, 2, 7, 5], np.int32)
    t = {"a": oracle.HostCol(a, "i32"), "b": oracle.HostCol(b, "i32")}
    r = oracle.groupby(t, ["a", "b"], [("count_star", None)])
    packed = [((int(x) & 0xFFFFFFFF) << 32 | (int(y) & 0xFFFFFFFF)) for x, y in zip(a, b)]
    packed = [p - (1 << 64) if p >= (1 << 63) else p for p in packed]
    assert r["keys"].tolist() == sorted(set(packed))
    assert r["vals"][0].tolist() == [2, 1, 1, 1]


def test_oracle_sum_i64_overflow_message(oracle):
    t = {"k": oracle.HostCol(np.zeros(2, np.int32), "i32"),
         "v": oracle.HostCol(np.array([2**62, 2**62], np.int64), "i64")}
    with pytest.raises(oracle.OracleError) as ei:
        oracle.groupby(t, ["k"], [("sum", "v")])
    assert "SUM(integer) overflow" in str(ei.value)


def test_oracle_compact_order(oracle):
    rng = np.random.default_rng(9)
    f = rng.integers(0, 100, 5000).astype(np.int32)
    rows = oracle.compact({"f": oracle.HostCol(f, "i32")}, [("f", "<", 50)])
    assert np.array_equal(rows, np.flatnonzero(f < 50).astype(np.uint32))


def test_oracle_sort_nulls_last_and_first(oracle):
    v = np.array([3, 1, 2, 1, 0], np.int32)
    valid = np.array([1, 0, 1, 1, 0], bool)
    bm = np.packbits(valid.astype(np.uint8), bitorder="little")
    last = oracle.sort_perm(oracle.HostCol(v, "i32", bm), False, False)
    first = oracle.sort_perm(oracle.HostCol(v, "i32", bm), False, True)
    assert last.tolist() == [3, 2, 0, 1, 4]
    assert first.tolist() == [1, 4, 3, 2, 0]
    assert unpack_bits(bm, 5).tolist() == valid.tolist()


def _same_groupby(r1: dict, r2: dict):
    assert r1["n_groups"] == r2["n_groups"]
    assert np.array_equal(r1["keys"], r2["keys"])
    assert np.array_equal(r1["key_null"], r2["key_null"])
    for a, b in zip(r1["vals"], r2["vals"]):
        assert np.array_equal(np.ascontiguousarray(a).view(np.uint8), np.ascontiguousarray(b).view(np.uint8))
    for a, b in zip(r1["valid"], r2["valid"]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("threads", [2, 7, 16])
def test_oracle_groupby_par_equals_sequential(oracle, threads):
    """The multi-threaded fold (key-range partitions, each in row order)
    gives bit-identical outputs to the sequential restatement: Zipf-skewed
    two-key groups with WHERE, f64 SUM/AVG, COUNT, int MIN/MAX."""
    rng = np.random.default_rng(5)
    n = 300_000
    ranks = np.minimum(rng.zipf(1.1, n), 50_000)
    a = (ranks * 7919 % 65536).astype(np.int32) - 30000
    b = (ranks * 104729 % 1000003).astype(np.int32)
    t = {"a": oracle.HostCol(a, "i32"), "b": oracle.HostCol(b, "i32"),
         "f": oracle.HostCol(rng.integers(0, 100, n).astype(np.int32), "i32"),
         "vd": oracle.HostCol(rng.normal(0, 1e3, n), "f64"),
         "vi": oracle.HostCol(rng.integers(-2**62, 2**62, n), "i64")}
    aggs = [("sum", "vd"), ("avg", "vd"), ("count_star", None), ("min", "vi"), ("max", "vi")]
    r1 = oracle.groupby(t, ["a", "b"], aggs, where=[("f", "<", 50)])
    r2 = oracle.groupby(t, ["a", "b"], aggs, where=[("f", "<", 50)], threads=threads)
    _same_groupby(r1, r2)


def test_oracle_groupby_par_null_keys_and_decimal(oracle):
    """Single key with NULLs (one NULL group, emitted last), nullable values,
    Decimal128 SUM: identical on many threads."""
    rng = np.random.default_rng(6)
    n = 200_000
    k = rng.integers(-500, 500, n).astype(np.int64)
    kv = rng.random(n) > 0.05
    v = rng.integers(-10**6, 10**6, n).astype(np.int64)
    vv = rng.random(n) > 0.1
    dec = np.stack([rng.integers(0, 10**9, n).astype(np.int64), np.zeros(n, np.int64)], axis=1)
    t = {"k": oracle.HostCol(k, "i64", np.packbits(kv.astype(np.uint8), bitorder="little")),
         "v": oracle.HostCol(v, "i64", np.packbits(vv.astype(np.uint8), bitorder="little")),
         "d": oracle.HostCol(dec, "dec128", scale=2)}
    aggs = [("sum", "v"), ("count", "v"), ("min", "v"), ("max", "v"), ("sum", "d"), ("count_star", None)]
    r1 = oracle.groupby(t, ["k"], aggs)
    r2 = oracle.groupby(t, ["k"], aggs, threads=8)
    _same_groupby(r1, r2)
    assert r2["key_null"][-1] and not r2["key_null"][:-1].any()


def test_oracle_groupby_par_overflow(oracle):
    """A group whose row-order i64 prefix leaves the range errors on every
    thread count, with the reference's message."""
    n = 50_000
    k = np.zeros(n, np.int32)
    k[n // 2:] = 1
    v = np.ones(n, np.int64)
    v[10] = 2**62
    v[11] = 2**62
    t = {"k": oracle.HostCol(k, "i32"), "v": oracle.HostCol(v, "i64")}
    for threads in (1, 4):
        with pytest.raises(oracle.OracleError) as ei:
            oracle.groupby(t, ["k"], [("sum", "v")], threads=threads)
        assert ei.value.status == oracle.OVERFLOW
        assert "SUM(integer) overflow" in str(ei.value)


@pytest.mark.parametrize("dt", ["i32", "i64"])
def test_hash_join_multi_matches_python_dict_join(oracle, dt):
    """The multi-match join against the reference's host join restated in
    Python (a dict from key to its build rows in ascending order, probed in
    row order), with duplicate keys, NULL keys on both sides and key -1; on
    unique keys it equals the unique-key oracle join."""
    rng = np.random.default_rng(31)
    nb, npr = 3000, 5000
    bk = rng.integers(-40, 400, nb).astype(np.int32 if dt == "i32" else np.int64)
    bk[::50] = -1
    pk = rng.integers(-60, 420, npr).astype(bk.dtype)
    bvalid = rng.random(nb) > 0.05
    pvalid = rng.random(npr) > 0.05
    table: dict[int, list[int]] = {}
    for i in range(nb):
        if bvalid[i]:
            table.setdefault(int(bk[i]), []).append(i)
    want_p, want_b = [], []
    for p in range(npr):
        if pvalid[p]:
            for b in table.get(int(pk[p]), []):
                want_p.append(p)
                want_b.append(b)

    def packbits(v):
        return np.packbits(v.astype(np.uint8), bitorder="little")

    op, ob = oracle.hash_join_multi(oracle.HostCol(bk, dt, packbits(bvalid)), oracle.HostCol(pk, dt, packbits(pvalid)))
    assert op.tolist() == want_p and ob.tolist() == want_b
    ub = rng.permutation(np.arange(-500, 500, dtype=bk.dtype))
    up, ubr = oracle.hash_join_multi(oracle.HostCol(ub, dt), oracle.HostCol(pk, dt))
    wp, wb = oracle.hash_join(oracle.HostCol(ub, dt), oracle.HostCol(pk, dt))
    assert np.array_equal(up, wp) and np.array_equal(ubr, wb)


def test_groupby_wide_matches_python_reduction(oracle):
    """The wide-key oracle against the reference's host wide reduction
    restated in Python: NULL-key rows dropped, wrapping int64 SUM, f64 SUM and
    AVG in row order, first-seen MIN / MAX, COUNT of valid inputs, groups in
    (key0, key1) order."""
    rng = np.random.default_rng(61)
    n = 20_000
    k0 = rng.integers(-5, 6, n).astype(np.int64) * (2 ** 40)
    k1 = rng.integers(-300, 300, n).astype(np.int32)
    vi = rng.integers(-2 ** 62, 2 ** 62, n)
    vd = rng.normal(0, 1e3, n)
    v32 = rng.integers(-1000, 1000, n).astype(np.int32)
    kv = rng.random(n) > 0.03
    vv = rng.random(n) > 0.2

    def bm(v):
        return np.packbits(v.astype(np.uint8), bitorder="little")

    table = {"k0": oracle.HostCol(k0, "i64", bm(kv)), "k1": oracle.HostCol(k1, "i32"),
             "vi": oracle.HostCol(vi, "i64", bm(vv)), "vd": oracle.HostCol(vd, "f64", bm(vv)),
             "v32": oracle.HostCol(v32, "i32")}
    aggs = [("sum", "vi"), ("sum", "vd"), ("avg", "v32"), ("count_star", None), ("count", "vi"),
            ("min", "vd"), ("max", "vi"), ("min", "v32")]
    r = oracle.groupby_wide(table, ["k0", "k1"], aggs)
    groups: dict = {}
    for i in range(n):
        if kv[i]:
            groups.setdefault((int(k0[i]), int(k1[i])), []).append(i)
    keys = sorted(groups)
    assert r["n_groups"] == len(keys)
    assert r["k0"].tolist() == [k[0] for k in keys] and r["k1"].tolist() == [k[1] for k in keys]
    for g, key in enumerate(keys):
        rows = groups[key]
        vrows = [i for i in rows if vv[i]]
        s = 0
        for i in vrows:
            s = (s + int(vi[i]) + 2 ** 63) % 2 ** 64 - 2 ** 63
        assert r["vals"][0][g] == s and r["valid"][0][g] == bool(vrows)
        fs = 0.0
        for i in vrows:
            fs += float(vd[i])
        assert (r["vals"][1][g] == fs) if vrows else not r["valid"][1][g]
        a = 0.0
        for i in rows:
            a += float(v32[i])
        assert r["vals"][2][g] == a / len(rows)
        assert r["vals"][3][g] == len(rows) and r["vals"][4][g] == len(vrows)
        if vrows:
            assert r["vals"][5][g] == min(float(vd[i]) for i in vrows)
            assert r["vals"][6][g] == max(int(vi[i]) for i in vrows)
        assert r["vals"][7][g] == min(int(v32[i]) for i in rows)


def test_groupby_wide_edge_cases(oracle):
    """No rows, every key NULL, and a group whose inputs are all NULL (NULL
    SUM / MIN / AVG, COUNT 0, COUNT(*) the row count)."""
    e = np.zeros(0, np.int64)
    r = oracle.groupby_wide({"a": oracle.HostCol(e, "i64"), "b": oracle.HostCol(e, "i64")}, ["a", "b"],
                            [("count_star", None)])
    assert r["n_groups"] == 0
    k = np.arange(8, dtype=np.int64)
    none = np.packbits(np.zeros(8, np.uint8), bitorder="little")
    r = oracle.groupby_wide({"a": oracle.HostCol(k, "i64", none), "b": oracle.HostCol(k, "i64")}, ["a", "b"],
                            [("count_star", None)])
    assert r["n_groups"] == 0
    v = np.array([5, 6, 7, 8, 9, 10, 11, 12], np.int64)
    vv = np.packbits(np.array([0, 0, 0, 0, 1, 1, 1, 1], np.uint8), bitorder="little")
    keys = np.array([1, 1, 1, 1, 2, 2, 2, 2], np.int64)
    t = {"a": oracle.HostCol(keys, "i64"), "b": oracle.HostCol(np.zeros(8, np.int32), "i32"),
         "v": oracle.HostCol(v, "i64", vv)}
    aggs = [("sum", "v"), ("min", "v"), ("avg", "v"), ("count", "v"), ("count_star", None)]
    r = oracle.groupby_wide(t, ["a", "b"], aggs)
    assert r["n_groups"] == 2 and r["k0"].tolist() == [1, 2]
    assert [x[0] for x in r["valid"]] == [False, False, False, True, True]
    assert [x[1] for x in r["valid"]] == [True] * 5
    assert [int(x[1]) if i != 2 else float(x[1]) for i, x in enumerate(r["vals"])] == [42, 9, 10.5, 4, 4]
    assert r["vals"][3][0] == 0 and r["vals"][4][0] == 4


@pytest.mark.parametrize("case", golden()["groupby_wide"], ids=lambda c: c["name"])
def test_oracle_groupby_wide_known_answers(oracle, case):
    """The wide-key oracle against the reference's own wide GROUP BY tests."""
    t = host_table(oracle, case["columns"])
    exp = case["expected"]
    r = oracle.groupby_wide(t, case["group_by"], [tuple(a) for a in case["aggs"]])
    assert r["k0"].tolist() == exp["k0"] and r["k1"].tolist() == exp["k1"]
    for a, want in enumerate(exp["aggs"]):
        assert r["vals"][a].tolist() == want and r["valid"][a].all()
