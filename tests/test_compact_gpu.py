"""GPU parity: bolt_compact / bolt_compact_mask against the oracle's
order-preserving filter (bit-exact rows and values). Both kernels are
covered: the bulk-staged one (columns on 16-byte boundaries, the default)
and the per-element one (FLAG_KERNEL_REGS, unaligned columns, wide rows)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from helpers import bitmap, unpack_bits

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kernel", ["bulk", "element"])
@pytest.mark.parametrize("n", [0, 1, 1000, 1023, 1024, 1025, 2047, 2048, 2049, 4095, 4096, 4097, 1_000_003,
                               1 << 22, (1 << 22) + 2047, 5_000_001])
def test_compact_predicate(bolt, engine, oracle, n, kernel):
    rng = np.random.default_rng(n)
    f = rng.integers(0, 100, n).astype(np.int32)
    x = rng.normal(0, 1, n)
    d = np.stack([rng.integers(0, 10**7, n), np.zeros(n, np.int64)], axis=1).astype(np.int64)
    xv = rng.random(n) > 0.1
    table = {"f": bolt.col(f, "i32").to("cuda"), "x": bolt.col(x, "f64", bitmap(xv)).to("cuda"),
             "d": bolt.col(d, "dec128").to("cuda")}
    flags = 0 if kernel == "bulk" else bolt.FLAG_KERNEL_REGS
    out, rows = engine.compact_columns(table, where=[("f", "<", 50)], flags=flags)
    want = oracle.compact({"f": oracle.HostCol(f, "i32")}, [("f", "<", 50)])
    assert np.array_equal(rows.cpu().numpy().view(np.uint32), want)
    assert np.array_equal(out["f"].numpy(), f[want])
    assert np.array_equal(out["x"].numpy().view(np.int64), x[want].view(np.int64))
    assert np.array_equal(out["d"].numpy(), d[want])
    assert np.array_equal(unpack_bits(out["x"].validity.cpu().numpy(), len(want)), xv[want])


@pytest.mark.parametrize("n", [300_000, (1 << 22) + 333])
def test_compact_float_predicate_and_conjunction(bolt, engine, oracle, n):
    rng = np.random.default_rng(5)
    x = rng.normal(0, 1, n)
    x[::50] = np.nan
    y = rng.integers(-10, 10, n).astype(np.int64)
    table = {"x": bolt.col(x, "f64").to("cuda"), "y": bolt.col(y, "i64").to("cuda")}
    where = [("x", ">=", -0.5), ("y", "!=", 0)]
    out, rows = engine.compact_columns(table, where=where)
    want = oracle.compact({"x": oracle.HostCol(x, "f64"), "y": oracle.HostCol(y, "i64")}, where)
    assert np.array_equal(rows.cpu().numpy().view(np.uint32), want)


@pytest.mark.parametrize("n", [500_000, (1 << 22) + 4097])
def test_compact_mask(bolt, engine, oracle, n):
    rng = np.random.default_rng(6)
    m = ((rng.random(n) < 0.3) * rng.integers(1, 256, n)).astype(np.uint8)  # any nonzero byte keeps
    v = rng.integers(0, 1 << 40, n).astype(np.int64)
    out, rows = engine.compact_columns({"v": bolt.col(v, "i64").to("cuda")}, mask=torch.from_numpy(m))
    idx = np.flatnonzero(m)
    assert np.array_equal(rows.cpu().numpy().view(np.uint32), idx.astype(np.uint32))
    assert np.array_equal(out["v"].numpy(), v[idx])


def test_compact_capacity_error(bolt, engine, oracle):
    f = np.zeros(10_000, np.int32)
    with pytest.raises(bolt.GpuCapacityError):
        engine.compact_columns({"f": bolt.col(f, "i32").to("cuda")}, where=[("f", "<", 50)], out_cap=100)


@pytest.mark.parametrize("n", [4095, 300_001, (1 << 22) + 1001])
def test_compact_wide_rows(bolt, engine, oracle, n):
    """56 bytes per row: the bulk kernel's 1,024-row tiles (one pass, and
    the two-pass form from 4,194,304 rows)."""
    rng = np.random.default_rng(n + 1)
    g = rng.integers(-5, 5, n).astype(np.int64)
    d1 = rng.integers(-(1 << 62), 1 << 62, (n, 2)).astype(np.int64)
    d2 = rng.integers(-(1 << 62), 1 << 62, (n, 2)).astype(np.int64)
    v = rng.integers(0, 1 << 30, n).astype(np.int64)
    table = {"g": bolt.col(g, "i64").to("cuda"), "d1": bolt.col(d1, "dec128").to("cuda"),
             "d2": bolt.col(d2, "dec128").to("cuda"), "v": bolt.col(v, "i64").to("cuda")}
    out, rows = engine.compact_columns(table, where=[("g", ">", 0)])
    want = oracle.compact({"g": oracle.HostCol(g, "i64")}, [("g", ">", 0)])
    assert np.array_equal(rows.cpu().numpy().view(np.uint32), want)
    for k, a in (("g", g), ("d1", d1), ("d2", d2), ("v", v)):
        assert np.array_equal(out[k].numpy(), a[want]), k


def test_compact_unaligned_columns(bolt, engine, oracle):
    """Columns that start 4 bytes past a 16-byte boundary take the
    per-element kernel."""
    rng = np.random.default_rng(11)
    n = 200_003
    f = rng.integers(0, 100, n + 1).astype(np.int32)
    v = rng.integers(0, 1 << 40, n + 1).astype(np.int64)
    ft = torch.from_numpy(f).cuda()[1:]
    vt = torch.from_numpy(v).cuda()[1:]
    table = {"f": bolt.Column(ft, "i32"), "v": bolt.Column(vt, "i64")}
    out, rows = engine.compact_columns(table, where=[("f", ">=", 30)])
    want = oracle.compact({"f": oracle.HostCol(f[1:], "i32")}, [("f", ">=", 30)])
    assert np.array_equal(rows.cpu().numpy().view(np.uint32), want)
    assert np.array_equal(out["f"].numpy(), f[1:][want])
    assert np.array_equal(out["v"].numpy(), v[1:][want])


@pytest.mark.parametrize("n", [3001, (1 << 22) + 5])
def test_compact_widest_rows(bolt, engine, oracle, n):
    """120 bytes per row (seven Decimal128 columns and an int64): 512-row
    tiles in both the one-pass and the two-pass form."""
    rng = np.random.default_rng(n + 2)
    g = rng.integers(0, 3, n).astype(np.int64)
    table = {"g": bolt.col(g, "i64").to("cuda")}
    decs = {}
    for i in range(7):
        decs[f"d{i}"] = rng.integers(-(1 << 62), 1 << 62, (n, 2)).astype(np.int64)
        table[f"d{i}"] = bolt.col(decs[f"d{i}"], "dec128").to("cuda")
    out, rows = engine.compact_columns(table, where=[("g", "==", 1)])
    want = oracle.compact({"g": oracle.HostCol(g, "i64")}, [("g", "==", 1)])
    assert np.array_equal(rows.cpu().numpy().view(np.uint32), want)
    assert np.array_equal(out["g"].numpy(), g[want])
    for k, a in decs.items():
        assert np.array_equal(out[k].numpy(), a[want]), k
