"""GPU parity: hash join build/probe and the fused join -> GROUP BY against
the oracle (bit-exact pairs in probe order, exact Decimal128 sums)."""

from __future__ import annotations

import importlib

import numpy as np
import pytest

from helpers import bitmap, golden, spec_arrays

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", golden()["join"], ids=lambda c: c["name"])
def test_join_known_answers(bolt, engine, oracle, case):
    bd, bv, bdt, _ = spec_arrays(case["build"])
    pd, pv, pdt, _ = spec_arrays(case["probe"])
    r = engine.hash_join_indices(bolt.col(bd, bdt, bv).to("cuda"), bolt.col(pd, pdt, pv).to("cuda"))
    pr, br = (x.cpu().numpy().view(np.uint32) for x in r)
    assert len(pr) == case["expected"]["n_pairs"]
    wp, wb = oracle.hash_join(oracle.HostCol(bd, bdt, bv), oracle.HostCol(pd, pdt, pv))
    assert np.array_equal(pr, wp) and np.array_equal(br, wb)


@pytest.mark.parametrize("dt", ["i32", "i64"])
def test_join_random_with_nulls(bolt, engine, oracle, dt):
    rng = np.random.default_rng(31)
    nb, npr = 50_000, 400_000
    bk = rng.permutation(1_000_000)[:nb].astype(np.int64) - 500_000
    if dt == "i64":
        bk = bk * 1_000_003
    pk = np.where(rng.random(npr) < 0.7, bk[rng.integers(0, nb, npr)], rng.integers(-2**40, 2**40, npr))
    bk = bk.astype(np.int32 if dt == "i32" else np.int64)
    pk = pk.astype(np.int32 if dt == "i32" else np.int64)
    bvalid = rng.random(nb) > 0.05
    pvalid = rng.random(npr) > 0.05
    b = bolt.col(bk, dt, bitmap(bvalid)).to("cuda")
    p = bolt.col(pk, dt, bitmap(pvalid)).to("cuda")
    pr, br = (x.cpu().numpy().view(np.uint32) for x in engine.hash_join_indices(b, p))
    wp, wb = oracle.hash_join(oracle.HostCol(bk, dt, bitmap(bvalid)), oracle.HostCol(pk, dt, bitmap(pvalid)))
    assert np.array_equal(pr, wp) and np.array_equal(br, wb)


def test_join_key_minus_one_and_duplicates(bolt, engine, oracle):
    b = np.array([-1, 4, 9], np.int64)
    p = np.array([9, -1, 3, -1, 4], np.int64)
    pr, br = (x.cpu().numpy().view(np.uint32) for x in
              engine.hash_join_indices(bolt.col(b, "i64").to("cuda"), bolt.col(p, "i64").to("cuda")))
    assert pr.tolist() == [0, 1, 3, 4] and br.tolist() == [2, 0, 0, 1]
    dup = np.array([1, 2, 1, 4, -1, 4], np.int64)
    pr, br = (x.cpu().numpy().view(np.uint32) for x in
              engine.hash_join_indices(bolt.col(dup, "i64").to("cuda"), bolt.col(p, "i64").to("cuda")))
    assert pr.tolist() == [1, 3, 4, 4] and br.tolist() == [4, 4, 3, 5]


def test_join_capacity_error(bolt, engine, oracle):
    b = np.arange(100, dtype=np.int64)
    p = np.tile(b, 10)
    with pytest.raises(bolt.GpuCapacityError):
        engine.hash_join_indices(bolt.col(b, "i64").to("cuda"), bolt.col(p, "i64").to("cuda"), out_cap=50)


@pytest.mark.parametrize("nb,npr", [(10_000, 200_000), (1_000_000, 4_000_000)])
def test_join_groupby_decimal(bolt, engine, oracle, nb, npr):
    """SELECT b.g, SUM(p.amount), COUNT(*) FROM p JOIN b ON p.fk = b.k GROUP BY b.g."""
    dg = importlib.import_module("craton_bolt_b200.datagen")
    bt = dg.join_build(nb, seed=3)
    pt = dg.join_probe(npr, nb, seed=3)
    g, s, c = engine.join_groupby(bolt.col(bt["k"], "i64").to("cuda"), bolt.col(bt["g"], "i32").to("cuda"),
                                  bolt.col(pt["fk"], "i64").to("cuda"),
                                  bolt.col(pt["amount"], "dec128", scale=2).to("cuda"))
    wg, wlo, whi, wc = oracle.join_groupby(oracle.HostCol(bt["k"], "i64"), bt["g"], oracle.HostCol(pt["fk"], "i64"),
                                           oracle.HostCol(pt["amount"], "dec128", scale=2))
    assert np.array_equal(g.numpy(), wg)
    sd = s.numpy()
    assert np.array_equal(sd[:, 0], wlo) and np.array_equal(sd[:, 1], whi)
    assert np.array_equal(c.numpy(), wc)
    assert s.scale == 2


def test_join_groupby_wide_decimal_and_overflow(bolt, engine, oracle):
    bk = np.arange(4, dtype=np.int64)
    bg = np.array([0, 1, 0, 1], np.int32)
    pk = np.array([0, 1, 2, 3, 0], np.int64)
    big = 10**30
    vals = [big, -5, big, 7, -3]
    lo = np.array([v & (2**64 - 1) for v in vals], np.uint64).view(np.int64)
    hi = np.array([(v >> 64) & (2**64 - 1) for v in vals], np.uint64).view(np.int64)
    amt = np.stack([lo, hi], axis=1)
    g, s, c = engine.join_groupby(bolt.col(bk, "i64").to("cuda"), bolt.col(bg, "i32").to("cuda"),
                                  bolt.col(pk, "i64").to("cuda"), bolt.col(amt, "dec128").to("cuda"))
    sd = s.numpy()
    got = [(int(h) << 64) | (int(l) & (2**64 - 1)) for l, h in sd]
    assert g.numpy().tolist() == [0, 1]
    assert got == [2 * big - 3, 2]
    assert c.numpy().tolist() == [3, 2]
    huge = 10**38 - 1
    lo = np.array([huge & (2**64 - 1)] * 2, np.uint64).view(np.int64)
    hi = np.array([huge >> 64] * 2, np.uint64).view(np.int64)
    with pytest.raises(bolt.TypeError_):
        engine.join_groupby(bolt.col(bk[:2], "i64").to("cuda"), bolt.col(np.zeros(2, np.int32), "i32").to("cuda"),
                            bolt.col(np.array([0, 1], np.int64), "i64").to("cuda"),
                            bolt.col(np.stack([lo, hi], axis=1), "dec128").to("cuda"))


def _join_groupby_vs_oracle(bolt, engine, oracle, bk, bg, pk, amt, kdt="i64", bvalid=None, pvalid=None):
    bkc = bolt.col(bk, kdt, bitmap(bvalid) if bvalid is not None else None).to("cuda")
    pkc = bolt.col(pk, kdt, bitmap(pvalid) if pvalid is not None else None).to("cuda")
    g, s, c = engine.join_groupby(bkc, bolt.col(bg, "i32").to("cuda"), pkc, bolt.col(amt, "dec128").to("cuda"))
    wg, wlo, whi, wc = oracle.join_groupby(
        oracle.HostCol(bk, kdt, bitmap(bvalid) if bvalid is not None else None), bg,
        oracle.HostCol(pk, kdt, bitmap(pvalid) if pvalid is not None else None), oracle.HostCol(amt, "dec128"))
    assert np.array_equal(g.numpy(), wg)
    sd = s.numpy()
    assert np.array_equal(sd[:, 0], wlo) and np.array_equal(sd[:, 1], whi)
    assert np.array_equal(c.numpy(), wc)


@pytest.mark.parametrize("span", ["narrow_negative", "full_int32"])
def test_join_groupby_payload_ranges(bolt, engine, oracle, span):
    """Group payloads in a narrow negative range and over the whole int32
    range (extremes included) equal the oracle."""
    rng = np.random.default_rng(21)
    nb, npr = 50_000, 400_000
    bk = rng.permutation(np.arange(-nb, nb, 2, dtype=np.int64) * 7919)
    if span == "narrow_negative":
        bg = rng.integers(-60, 40, len(bk)).astype(np.int32)
    else:
        pool = np.array([-(2**31), 2**31 - 1, 0, -1, 123456789], np.int32)
        bg = pool[rng.integers(0, len(pool), len(bk))]
    pk = np.where(rng.random(npr) < 0.8, bk[rng.integers(0, len(bk), npr)], rng.integers(-(2**40), 2**40, npr))
    amt = np.stack([rng.integers(0, 10**7, npr), np.zeros(npr, np.int64)], axis=1).astype(np.int64)
    _join_groupby_vs_oracle(bolt, engine, oracle, bk, bg, pk, amt)


@pytest.mark.parametrize("kdt", ["i32", "i64"])
def test_join_groupby_extreme_keys_and_nulls(bolt, engine, oracle, kdt):
    """Keys -1, 0 and the dtype's extremes, NULL build and probe keys."""
    rng = np.random.default_rng(22)
    info = np.iinfo(np.int32 if kdt == "i32" else np.int64)
    special = np.array([-1, 0, info.min, info.max, 1, -2], dtype=np.int64)
    rest = rng.choice(np.arange(10, 200_000, dtype=np.int64), 20_000, replace=False)
    bk = np.concatenate([special, rest]).astype(np.int32 if kdt == "i32" else np.int64)
    bg = rng.integers(0, 7, len(bk)).astype(np.int32)
    npr = 150_000
    pk = bk[rng.integers(0, len(bk), npr)].copy()
    pk[::97] = -5  # absent
    bvalid = rng.random(len(bk)) > 0.05
    pvalid = rng.random(npr) > 0.05
    amt = np.stack([rng.integers(-10**6, 10**6, npr), np.zeros(npr, np.int64)], axis=1).astype(np.int64)
    amt[:, 1] = amt[:, 0] >> 63
    _join_groupby_vs_oracle(bolt, engine, oracle, bk, bg, pk, amt, kdt, bvalid, pvalid)


@pytest.mark.parametrize("kdt", ["i32", "i64"])
def test_join_groupby_table_larger_than_l2(bolt, engine, oracle, kdt):
    """A 3M-key build side (8M slots, 128 MB table, larger than L2) probed by
    12M rows: keys -1, 0 and the dtype's extremes, 10 % absent probe keys;
    equals the oracle exactly."""
    rng = np.random.default_rng(23)
    nb, npr = 3_000_000, 12_000_000
    info = np.iinfo(np.int32 if kdt == "i32" else np.int64)
    special = np.array([-1, 0, info.min, info.max], dtype=np.int64)
    if kdt == "i32":  # an odd multiplier permutes [0, 2^31)
        rest = (np.arange(1, nb + 1, dtype=np.int64) * 2654435761) % (2**31)
    else:  # ... and [0, 2^64)
        rest = (np.arange(1, nb + 1, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15)).view(np.int64)
    rest = np.setdiff1d(rest, special)[: nb - len(special)]
    bk = rng.permutation(np.concatenate([special, rest])).astype(np.int32 if kdt == "i32" else np.int64)
    bg = rng.integers(0, 1000, len(bk)).astype(np.int32)
    pk = bk[rng.integers(0, len(bk), npr)].copy()
    absent = rng.random(npr) < 0.1
    pk[absent] = -2  # never a build key (the build keys are -1, 0, extremes and non-negative values)
    amt = np.stack([rng.integers(-10**9, 10**9, npr), np.zeros(npr, np.int64)], axis=1).astype(np.int64)
    amt[:, 1] = amt[:, 0] >> 63
    assert -2 not in set(special.tolist())
    _join_groupby_vs_oracle(bolt, engine, oracle, bk, bg, pk, amt, kdt)


@pytest.mark.parametrize("dt", ["i32", "i64"])
@pytest.mark.parametrize("shape", ["few_repeats", "heavy_key", "with_nulls"])
def test_join_duplicate_build_keys(bolt, engine, oracle, dt, shape):
    """Build keys that repeat (the reference's collision-list path): every
    matching build row pairs with the probe row, in probe order and then
    ascending build row, exactly as the reference's host join map; the
    output grows past the probe length (the wrapper re-sizes it once)."""
    rng = np.random.default_rng({"few_repeats": 51, "heavy_key": 52, "with_nulls": 53}[shape])
    nb, npr = 400_000, 300_000
    bk = rng.integers(0, 150_000, nb).astype(np.int32 if dt == "i32" else np.int64)
    bk[::1000] = -1
    if shape == "heavy_key":
        bk[rng.random(nb) < 0.05] = 7  # one key with ~20,000 build rows
    pk = rng.integers(-1000, 160_000, npr).astype(bk.dtype)
    pk[::997] = -1
    if shape == "heavy_key":
        pk[::5000] = 7
    bvalid = rng.random(nb) > 0.05 if shape == "with_nulls" else None
    pvalid = rng.random(npr) > 0.05 if shape == "with_nulls" else None
    b = bolt.col(bk, dt, bitmap(bvalid) if bvalid is not None else None).to("cuda")
    p = bolt.col(pk, dt, bitmap(pvalid) if pvalid is not None else None).to("cuda")
    pr, br = (x.cpu().numpy().view(np.uint32) for x in engine.hash_join_indices(b, p))
    wp, wb = oracle.hash_join_multi(oracle.HostCol(bk, dt, bitmap(bvalid) if bvalid is not None else None),
                                    oracle.HostCol(pk, dt, bitmap(pvalid) if pvalid is not None else None))
    assert len(wp) > npr
    assert np.array_equal(pr, wp) and np.array_equal(br, wb)
    # The fused join -> GROUP BY needs one build row per key: it declines.
    assert engine.join_groupby(b, bolt.col(np.zeros(nb, np.int32), "i32").to("cuda"), p,
                               bolt.col(np.zeros((npr, 2), np.int64), "dec128").to("cuda")) is None
