"""GPU: batched (one persistent launch) and served (continuous batching)
filter + GROUP BY. Every query's result must equal the oracle's, and be
bit-identical to the same query run alone."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from helpers import compare_groupby

pytestmark = pytest.mark.gpu


def make_table(bolt, n, seed):
    rng = np.random.default_rng(seed)
    t = {
        "k32": rng.integers(0, 1 << 31, n).astype(np.int32),
        "k64": rng.integers(-(1 << 62), 1 << 62, n).astype(np.int64),
        "vi": rng.integers(-10**9, 10**9, n).astype(np.int64),
        "vd": rng.normal(0, 1e3, n),
        "f": rng.integers(0, 100, n).astype(np.int32),
    }
    dts = {"k32": "i32", "k64": "i64", "vi": "i64", "vd": "f64", "f": "i32"}
    dev = {k: bolt.col(v, dts[k]).to("cuda") for k, v in t.items()}
    return t, dts, dev


def query_specs(n_rows, n_q, seed):
    """Queries of uneven sizes and cardinalities over one resident table:
    key = k % card (via a derived column), filter f < t."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_q):
        rows = int(np.exp(rng.uniform(np.log(1000), np.log(n_rows))))
        begin = int(rng.integers(0, n_rows - rows + 1))
        card = int(np.exp(rng.uniform(np.log(10), np.log(200_000))))
        key = "k32" if i % 2 == 0 else "k64"
        val = "vi" if i % 3 else "vd"
        out.append(dict(begin=begin, end=begin + rows, card=card, key=key, val=val, t=int(rng.integers(10, 100))))
    return out


def keyed_columns(bolt, t, dts, specs):
    """One derived key column per distinct (key, card): key % card."""
    cols = {}
    for s in specs:
        name = f"{s['key']}_{s['card']}"
        if name not in cols:
            a = t[s["key"]] % s["card"]
            cols[name] = (a.astype(np.int32 if s["key"] == "k32" else np.int64), dts[s["key"]])
    return {k: bolt.col(v, d).to("cuda") for k, (v, d) in cols.items()}, cols


def test_batch_matches_alone_and_oracle(bolt, engine, oracle):
    n = 400_000
    t, dts, dev = make_table(bolt, n, 1)
    specs = query_specs(n, 40, 2)
    kdev, khost = keyed_columns(bolt, t, dts, specs)
    prepared, alone = [], []
    for s in specs:
        kname = f"{s['key']}_{s['card']}"
        table = {kname: kdev[kname], s["val"]: dev[s["val"]], "f": dev["f"]}
        aggs = [("sum", s["val"]), ("count_star", None), ("max", s["val"])]
        where = [("f", "<", s["t"])]
        prepared.append(engine.prepare_groupby(table, [kname], aggs, where, groups_hint=s["card"],
                                               rows=(s["begin"], s["end"])))
    results = engine.execute_batch(prepared)
    for s, r in zip(specs, results):
        kname = f"{s['key']}_{s['card']}"
        sl = slice(s["begin"], s["end"])
        host = {kname: oracle.HostCol(khost[kname][0][sl], khost[kname][1]),
                s["val"]: oracle.HostCol(t[s["val"]][sl], dts[s["val"]]), "f": oracle.HostCol(t["f"][sl], "i32")}
        aggs = [("sum", s["val"]), ("count_star", None), ("max", s["val"])]
        orc = oracle.groupby(host, [kname], aggs, where=[("f", "<", s["t"])])
        compare_groupby(r, orc, [khost[kname][1]], aggs, [dts[s["val"]], None, dts[s["val"]]])
        # alone: same rows as their own columns
        a = engine.execute_groupby({kname: bolt.Column(kdev[kname].data[sl], kdev[kname].dtype),
                                    s["val"]: bolt.Column(dev[s["val"]].data[sl], dts[s["val"]]),
                                    "f": bolt.Column(dev["f"].data[sl], "i32")}, [kname], aggs,
                                   where=[("f", "<", s["t"])], groups_hint=s["card"])
        for x, y in zip(r.aggs + r.keys, a.aggs + a.keys):
            xa = x.data.view(torch.int64) if x.data.dtype == torch.float64 else x.data
            ya = y.data.view(torch.int64) if y.data.dtype == torch.float64 else y.data
            assert torch.equal(xa, ya), "batched result differs from the query run alone"


def test_batch_recovers_undersized_hint(bolt, engine, oracle):
    n = 200_000
    t, dts, dev = make_table(bolt, n, 3)
    k = (t["k32"] % 50_000).astype(np.int32)
    kd = bolt.col(k, "i32").to("cuda")
    pq = [engine.prepare_groupby({"k": kd, "vi": dev["vi"]}, ["k"], [("sum", "vi")], groups_hint=10,
                                 out_cap=60_000, rows=(0, n)),
          engine.prepare_groupby({"k": kd, "vi": dev["vi"]}, ["k"], [("count_star", None)], groups_hint=50_000,
                                 rows=(0, n // 2))]
    r = engine.execute_batch(pq)
    orc = oracle.groupby({"k": oracle.HostCol(k, "i32"), "vi": oracle.HostCol(t["vi"], "i64")}, ["k"], [("sum", "vi")])
    compare_groupby(r[0], orc, ["i32"], [("sum", "vi")], ["i64"])
    assert r[1].n_groups == len(np.unique(k[: n // 2]))


def test_batch_graph_replay(bolt, engine, oracle):
    """A captured batch graph replays to the same results, and follows
    in-place updates of its columns."""
    n = 200_000
    t, dts, dev = make_table(bolt, n, 9)
    specs = query_specs(n, 12, 10)
    kdev, khost = keyed_columns(bolt, t, dts, specs)
    prepared = []
    for s in specs:
        kname = f"{s['key']}_{s['card']}"
        table = {kname: kdev[kname], s["val"]: dev[s["val"]], "f": dev["f"]}
        prepared.append(engine.prepare_groupby(table, [kname], [("sum", s["val"]), ("count_star", None)],
                                               [("f", "<", s["t"])], groups_hint=s["card"],
                                               rows=(s["begin"], s["end"])))
    g = bolt.BatchGraph(0, prepared)
    try:
        g.launch()
        r1 = [[c.data.clone() for c in (r.keys + r.aggs)] for r in g.results()]
        g.launch()
        r2 = [[c.data.clone() for c in (r.keys + r.aggs)] for r in g.results()]
        for a, b in zip(r1, r2):
            for x, y in zip(a, b):
                assert torch.equal(x, y)
        for s, r in zip(specs, g.results()):
            kname = f"{s['key']}_{s['card']}"
            sl = slice(s["begin"], s["end"])
            host = {kname: oracle.HostCol(khost[kname][0][sl], khost[kname][1]),
                    s["val"]: oracle.HostCol(t[s["val"]][sl], dts[s["val"]]), "f": oracle.HostCol(t["f"][sl], "i32")}
            aggs = [("sum", s["val"]), ("count_star", None)]
            orc = oracle.groupby(host, [kname], aggs, where=[("f", "<", s["t"])])
            compare_groupby(r, orc, [khost[kname][1]], aggs, [dts[s["val"]], None])
        # In-place update of the filter column: replay sees the new data.
        dev["f"].data.fill_(0)
        g.launch()
        for s, r in zip(specs, g.results()):
            assert int(r.aggs[1].data.sum()) == s["end"] - s["begin"]
    finally:
        g.close()


@pytest.mark.parametrize("n,n_q,lanes,burst", [(300_000, 60, 2, False), (12_000_000, 24, 4, False),
                                               (300_000, 200, 4, True), (12_000_000, 40, 3, True)])
def test_server_mix_equals_alone(bolt, engine, oracle, n, n_q, lanes, burst):
    """Served results equal the query run alone. The larger table gives
    queries above the size that is admitted alone, and several lanes run
    different kernels and shared-memory sizes concurrently. `burst` submits
    all queries in one bolt_server_submit_batch call, so lanes form full
    batches."""
    t, dts, dev = make_table(bolt, n, 5)
    specs = query_specs(n, n_q, 6)
    kdev, khost = keyed_columns(bolt, t, dts, specs)
    srv = bolt.Server(0, scratch_bytes=4 << 30, max_batch=16, n_lanes=lanes)
    try:
        tickets, pqs = [], []
        for s in specs:
            kname = f"{s['key']}_{s['card']}"
            table = {kname: kdev[kname], s["val"]: dev[s["val"]], "f": dev["f"]}
            pq = engine.prepare_groupby(table, [kname], [("sum", s["val"]), ("count_star", None)],
                                        [("f", "<", s["t"])], groups_hint=s["card"], rows=(s["begin"], s["end"]))
            pqs.append((pq, s, kname))
        if burst:
            ts = srv.submit_many([pq for pq, _, _ in pqs])
            tickets = [(t, s, kname) for t, (_, s, kname) in zip(ts, pqs)]
        else:
            tickets = [(srv.submit(pq), s, kname) for pq, s, kname in pqs]
        lat = []
        for ticket, s, kname in tickets:
            r, us = srv.wait(ticket)
            lat.append(us)
            sl = slice(s["begin"], s["end"])
            a = engine.execute_groupby({kname: bolt.Column(kdev[kname].data[sl], kdev[kname].dtype),
                                        s["val"]: bolt.Column(dev[s["val"]].data[sl], dts[s["val"]]),
                                        "f": bolt.Column(dev["f"].data[sl], "i32")}, [kname],
                                       [("sum", s["val"]), ("count_star", None)], where=[("f", "<", s["t"])],
                                       groups_hint=s["card"])
            assert r.n_groups == a.n_groups
            for x, y in zip(r.aggs + r.keys, a.aggs + a.keys):
                xa = x.data.view(torch.int64) if x.data.dtype == torch.float64 else x.data
                ya = y.data.view(torch.int64) if y.data.dtype == torch.float64 else y.data
                assert torch.equal(xa, ya), "served result differs from the query run alone"
        assert all(v > 0 for v in lat)
    finally:
        srv.close()
