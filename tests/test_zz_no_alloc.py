"""GPU: bolt_groupby_noalloc, the GROUP BY that allocates no device memory.

It serves callers that may not call cudaMalloc / cudaFree: an engine whose
own pool allocator owns all of HBM, or a latency-critical loop where an
allocation would synchronise the device. Its scratch is a fixed array inside
the library that every call reuses, so these tests check, through the C ABI,
that two calls in a row (the second one meeting the first one's leftovers in
that array) return what the allocating entry point bolt_groupby returns, and
that a query beyond the array's limit is refused with a clear message.

The file sorts last so that a failure here never hides the other GPU tests;
it also passes when run alone in a fresh process.
"""

from __future__ import annotations

import ctypes as C

import numpy as np
import pytest
import torch

from helpers import REL_TOL, assert_float_close, bitmap

pytestmark = pytest.mark.gpu

ERR_CAPACITY = 4


def make_table(bolt, n, n_keys, seed):
    rng = np.random.default_rng(seed)
    k = rng.integers(-n_keys // 2, n_keys // 2, n).astype(np.int32)
    k2 = rng.integers(0, 3, n).astype(np.int32)
    f = rng.integers(0, 100, n).astype(np.int32)
    vi = rng.integers(-10**9, 10**9, n).astype(np.int64)
    vd = rng.normal(0, 1e3, n)
    vdv = rng.random(n) > 0.1
    return {"k": bolt.col(k, "i32").to("cuda"), "k2": bolt.col(k2, "i32").to("cuda"),
            "f": bolt.col(f, "i32").to("cuda"), "vi": bolt.col(vi, "i64").to("cuda"),
            "vd": bolt.col(vd, "f64", bitmap(vdv)).to("cuda")}


def run_noalloc(bolt, pq):
    err = C.create_string_buffer(256)
    stream = torch.cuda.current_stream().cuda_stream
    st = bolt.lib().bolt_groupby_noalloc(C.byref(pq.desc), C.byref(pq.out), C.c_void_p(stream), err, 256)
    return st, err.value.decode()


def assert_same(got, want):
    """Output of the allocation-free call vs bolt_groupby: keys, counts,
    integer aggregates and validity exactly; float64 within REL_TOL."""
    assert got.n_groups == want.n_groups
    for g, w in zip(got.keys + got.aggs, want.keys + want.aggs):
        assert g.dtype == w.dtype
        np.testing.assert_array_equal(g.valid_mask(), w.valid_mask())
        ok = w.valid_mask()
        if g.dtype == "f64":
            assert_float_close(g.numpy()[ok], w.numpy()[ok], REL_TOL, "f64 aggregate")
        else:
            np.testing.assert_array_equal(g.numpy()[ok], w.numpy()[ok])


QUERIES = [
    # (rows, groups hint, distinct keys, seed, group by, aggregates, where)
    (1_000_000, 4000, 4000, 31, ["k"],
     [("sum", "vi"), ("count_star", None), ("min", "vi"), ("max", "vi"), ("sum", "vd"), ("avg", "vd"),
      ("count", "vd")], []),
    (300_000, 1500, 500, 32, ["k", "k2"], [("count_star", None), ("sum", "vd"), ("max", "vd")], [("f", "<", 40)]),
]


def test_noalloc_matches_groupby_on_two_calls_in_a_row(bolt, engine):
    """Two different queries back to back (the second has fewer groups and
    other aggregates, so leftovers of the first would show), each compared
    with bolt_groupby on the same input."""
    for rows, hint, nk, seed, group_by, aggs, where in QUERIES:
        table = make_table(bolt, rows, nk, seed)
        want = engine.execute_groupby(table, group_by, aggs, where=where, groups_hint=hint)
        pq = engine.prepare_groupby(table, group_by, aggs, where, groups_hint=hint, out_cap=8192)
        st, msg = run_noalloc(bolt, pq)
        assert st == 0, msg
        assert_same(pq.result(False), want)


def test_noalloc_repeated_call_gives_the_same_result(bolt, engine):
    rows, hint, nk, seed, group_by, aggs, where = QUERIES[0]
    table = make_table(bolt, rows, nk, seed)
    want = engine.execute_groupby(table, group_by, aggs, where=where, groups_hint=hint)
    for _ in range(2):
        pq = engine.prepare_groupby(table, group_by, aggs, where, groups_hint=hint, out_cap=8192)
        st, msg = run_noalloc(bolt, pq)
        assert st == 0, msg
        assert_same(pq.result(False), want)


def test_noalloc_refuses_more_groups_than_its_table_holds(bolt, engine):
    table = make_table(bolt, 200_000, 20_000, 33)
    pq = engine.prepare_groupby(table, ["k"], [("count_star", None)], [], groups_hint=0, out_cap=1 << 15)
    st, msg = run_noalloc(bolt, pq)
    assert st == ERR_CAPACITY
    assert "6144 groups" in msg


def test_noalloc_grows_past_a_low_hint(bolt, engine):
    """A hint far below the real group count (10 vs about 3000) starts with a
    small table; the call grows it within the array and returns what
    bolt_groupby returns."""
    table = make_table(bolt, 400_000, 3000, 34)
    aggs = [("count_star", None), ("sum", "vi"), ("min", "vi"), ("max", "vd")]
    want = engine.execute_groupby(table, ["k"], aggs, groups_hint=3000)
    assert want.n_groups > 2500
    pq = engine.prepare_groupby(table, ["k"], aggs, [], groups_hint=10, out_cap=8192)
    st, msg = run_noalloc(bolt, pq)
    assert st == 0, msg
    assert_same(pq.result(False), want)


def test_noalloc_output_capacity_below_the_group_count(bolt, engine):
    table = make_table(bolt, 100_000, 2000, 35)
    pq = engine.prepare_groupby(table, ["k"], [("count_star", None)], [], groups_hint=2000, out_cap=100)
    st, msg = run_noalloc(bolt, pq)
    assert st == ERR_CAPACITY
    assert "capacity" in msg
