"""GPU parity: bolt_compact / bolt_compact_mask against the oracle's
order-preserving filter (bit-exact rows and values)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from helpers import bitmap, unpack_bits

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n", [0, 1, 1000, 1023, 1024, 1025, 2048, 2049, 1_000_003])
def test_compact_predicate(bolt, engine, oracle, n):
    rng = np.random.default_rng(n)
    f = rng.integers(0, 100, n).astype(np.int32)
    x = rng.normal(0, 1, n)
    d = np.stack([rng.integers(0, 10**7, n), np.zeros(n, np.int64)], axis=1).astype(np.int64)
    xv = rng.random(n) > 0.1
    table = {"f": bolt.col(f, "i32").to("cuda"), "x": bolt.col(x, "f64", bitmap(xv)).to("cuda"),
             "d": bolt.col(d, "dec128").to("cuda")}
    out, rows = engine.compact_columns(table, where=[("f", "<", 50)])
    want = oracle.compact({"f": oracle.HostCol(f, "i32")}, [("f", "<", 50)])
    assert np.array_equal(rows.cpu().numpy().view(np.uint32), want)
    assert np.array_equal(out["f"].numpy(), f[want])
    assert np.array_equal(out["x"].numpy().view(np.int64), x[want].view(np.int64))
    assert np.array_equal(out["d"].numpy(), d[want])
    assert np.array_equal(unpack_bits(out["x"].validity.cpu().numpy(), len(want)), xv[want])


def test_compact_float_predicate_and_conjunction(bolt, engine, oracle):
    rng = np.random.default_rng(5)
    n = 300_000
    x = rng.normal(0, 1, n)
    x[::50] = np.nan
    y = rng.integers(-10, 10, n).astype(np.int64)
    table = {"x": bolt.col(x, "f64").to("cuda"), "y": bolt.col(y, "i64").to("cuda")}
    where = [("x", ">=", -0.5), ("y", "!=", 0)]
    out, rows = engine.compact_columns(table, where=where)
    want = oracle.compact({"x": oracle.HostCol(x, "f64"), "y": oracle.HostCol(y, "i64")}, where)
    assert np.array_equal(rows.cpu().numpy().view(np.uint32), want)


def test_compact_mask(bolt, engine, oracle):
    rng = np.random.default_rng(6)
    n = 500_000
    m = (rng.random(n) < 0.3).astype(np.uint8)
    v = rng.integers(0, 1 << 40, n).astype(np.int64)
    out, rows = engine.compact_columns({"v": bolt.col(v, "i64").to("cuda")}, mask=torch.from_numpy(m))
    idx = np.flatnonzero(m)
    assert np.array_equal(rows.cpu().numpy().view(np.uint32), idx.astype(np.uint32))
    assert np.array_equal(out["v"].numpy(), v[idx])


def test_compact_capacity_error(bolt, engine, oracle):
    f = np.zeros(10_000, np.int32)
    with pytest.raises(bolt.GpuCapacityError):
        engine.compact_columns({"f": bolt.col(f, "i32").to("cuda")}, where=[("f", "<", 50)], out_cap=100)
