"""GPU parity: bolt_radix_sort_perm (ORDER BY permutation) against the oracle,
bit-exact, including stability, NULL placement and float specials."""

from __future__ import annotations

import importlib

import numpy as np
import pytest
import torch

from helpers import bitmap, golden

pytestmark = pytest.mark.gpu


def gpu_perm(bolt, engine, data, dt, valid=None, desc=False, nulls_first=False):
    c = bolt.col(data, dt, valid).to("cuda")
    return engine.sort_indices([c], desc, nulls_first).cpu().numpy().view(np.uint32)


def check(bolt, engine, oracle, data, dt, valid=None, desc=False, nulls_first=False):
    got = gpu_perm(bolt, engine, data, dt, valid, desc, nulls_first)
    want = oracle.sort_perm(oracle.HostCol(data, dt, valid), desc, nulls_first)
    assert np.array_equal(got, want), f"first diff at {np.flatnonzero(got != want)[:5]}"
    return got


def sort_input(oracle, case):
    n = case["n"]
    if case["gen"] == "shuffle_iota":
        return oracle.shuffle_deterministic(np.arange(n, dtype=np.uint32), case["seed"]).view(np.int32).copy()
    if case["gen"] == "mul7919_mod_shuffle":
        base = (np.arange(n, dtype=np.int64) * 7919) % 1_000_000
        idx = oracle.shuffle_deterministic(np.arange(n, dtype=np.uint32), case["seed"]).astype(np.int64)
        return base[idx]
    return np.sin(np.arange(n, dtype=np.float64) * 1.61803398875)


@pytest.mark.parametrize("case", golden()["sort"], ids=lambda c: c["name"])
def test_sort_known_answers(bolt, engine, oracle, case):
    v = sort_input(oracle, case)
    perm = check(bolt, engine, oracle, v, case["dtype"], desc=case["descending"])
    want = np.sort(v)[::-1] if case["descending"] else np.sort(v)
    assert np.array_equal(v[perm], want)


@pytest.mark.parametrize("dt", ["i32", "i64", "f32", "f64", "u32"])
@pytest.mark.parametrize("desc", [False, True])
def test_sort_dtypes_with_duplicates(bolt, engine, oracle, dt, desc):
    rng = np.random.default_rng(hash((dt, desc)) % 2**32)
    n = 300_001
    if dt in ("f32", "f64"):
        v = rng.normal(0, 1e3, n).round(1).astype(np.float32 if dt == "f32" else np.float64)
        v[::97] = -0.0
        v[::89] = 0.0
        v[::101] = np.inf
        v[::103] = -np.inf
        v[::107] = np.nan
    elif dt == "u32":
        v = rng.integers(0, 5000, n).astype(np.uint32)
    else:
        v = rng.integers(-5000, 5000, n).astype(np.int32 if dt == "i32" else np.int64)
    check(bolt, engine, oracle, v, dt, desc=desc)


def test_sort_f32_specials_nan_payloads(bolt, engine, oracle):
    dg = importlib.import_module("craton_bolt_b200.datagen")
    v = dg.sort_f32(1_000_000, seed=5, nan_frac=0.001)
    got = check(bolt, engine, oracle, v, "f32")
    s = v[got]
    n_nan = int(np.isnan(v).sum())
    assert n_nan > 0 and np.isnan(s[-n_nan:]).all()


def test_sort_i64_full_range_large(bolt, engine, oracle):
    dg = importlib.import_module("craton_bolt_b200.datagen")
    v = dg.sort_i64(4_000_000, seed=4)
    check(bolt, engine, oracle, v, "i64")


@pytest.mark.parametrize("nulls_first", [False, True])
def test_sort_nulls(bolt, engine, oracle, nulls_first):
    rng = np.random.default_rng(21)
    n = 100_000
    v = rng.integers(-100, 100, n).astype(np.int32)
    valid = rng.random(n) > 0.2
    check(bolt, engine, oracle, v, "i32", bitmap(valid), nulls_first=nulls_first)


def test_sort_multi_key(bolt, engine, oracle):
    rng = np.random.default_rng(22)
    n = 200_000
    a = rng.integers(0, 50, n).astype(np.int32)
    b = rng.normal(0, 1, n).round(2)
    c = rng.integers(0, 3, n).astype(np.int64)
    cv = rng.random(n) > 0.1
    cols = [bolt.col(a, "i32").to("cuda"), bolt.col(b, "f64").to("cuda"), bolt.col(c, "i64", bitmap(cv)).to("cuda")]
    desc, nf = [False, True, False], [False, False, True]
    got = engine.sort_indices(cols, desc, nf).cpu().numpy().view(np.uint32)
    want = oracle.sort_perm([oracle.HostCol(a, "i32"), oracle.HostCol(b, "f64"), oracle.HostCol(c, "i64", bitmap(cv))],
                            desc, nf)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("n", [0, 1, 2, 3071, 3072, 3073, 9217, 65537])
def test_sort_edge_sizes(bolt, engine, oracle, n):
    """Tile boundaries of 64-bit keys (3,072 keys per tile)."""
    v = np.random.default_rng(n).integers(-3, 3, n).astype(np.int64)
    check(bolt, engine, oracle, v, "i64")


@pytest.mark.parametrize("dt", ["i32", "f32"])
@pytest.mark.parametrize("n", [5119, 5120, 5121, 15361, 65537])
def test_sort_edge_sizes_32bit(bolt, engine, oracle, n, dt):
    """Tile boundaries of 32-bit keys (5,120 keys per tile)."""
    v = np.random.default_rng(n).integers(-3, 3, n)
    check(bolt, engine, oracle, v.astype(np.int32 if dt == "i32" else np.float32), dt)


def test_sort_constant_keys_is_identity(bolt, engine, oracle):
    v = np.full(50_000, 7, np.int64)
    got = check(bolt, engine, oracle, v, "i64")
    assert np.array_equal(got, np.arange(50_000, dtype=np.uint32))
