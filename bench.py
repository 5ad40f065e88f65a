#!/usr/bin/env python
"""Benchmark of the B200 relational hot path (one JSON line on rank 0).

Default workload (`--workload groupby_filtered`): the filtered
high-cardinality two-key GROUP BY
  SELECT a, b, SUM(vd), AVG(vd), COUNT(*), MIN(vi), MAX(vi)
  FROM t WHERE f < 50 GROUP BY a, b
over 100,000,000 seeded synthetic rows ((a, b) int32 pairs of 10M Zipf(1.1)
ranks, f int32 U[0,100), vd f64 N(0,1e3), vi int64 uniform).

At N=1 the default line also carries an `operators` map: every other
workload below at its full size with fewer repeats. Other workloads
(per-operator lines): groupby_plain (1M rows, 1024 keys),
join_groupby (10M-row build, 200M-row probe, Decimal128 SUM), sort_i64
(256M int64 keys), sort_f32 (64M float32 keys with specials), compact
(100M-row WHERE compaction), batch (4096 filter + GROUP BY queries,
batched / served vs one at a time).

  value      rows/s (queries/s for batch) with inputs resident in HBM,
             device-timed over K steps (CUDA events on the launch stream)
  e2e        the same metric through the public API from pinned host
             columns, host->device copies and result readback timed
  roofline   the dominant kernel's algorithmic bytes / its CUDA-event time
  cpu_baseline  the CPU restatement of the reference's host path (oracle)
             on a bounded sample of the same rows

`--impl reference` times the CPU restatement of the reference's host path
(the reference itself is Rust and cannot be built here) on the workload and
prints the same line with "impl": "reference". Multi-GPU (torchrun): the
path is run as independent replicas, one per rank; value sums all ranks'
rows over the max per-rank device time.
"""

from __future__ import annotations

import argparse
import ctypes as C
import gc
import importlib
import importlib.util
import json
import math
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

import faulthandler

faulthandler.enable()  # a native crash prints every thread's Python stack to stderr

REPO = Path(__file__).resolve().parent


def progress(msg: str):
    """Progress marker on stderr (stdout carries only the JSON line)."""
    sys.stderr.write(f"[bench {time.strftime('%H:%M:%S')}] {msg}\n")
    sys.stderr.flush()


METRIC = "rows/s & HBM GB/s (of ~8 TB/s) per operator; batched q/s + p99 vs per-query"


def load_package():
    name = "craton_bolt_b200"
    if name in sys.modules:
        return sys.modules[name]
    pkg = REPO / "craton-bolt_b200"
    spec = importlib.util.spec_from_file_location(name, pkg / "__init__.py", submodule_search_locations=[str(pkg)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def datagen():
    load_package()
    return importlib.import_module("craton_bolt_b200.datagen")


def oracle_mod():
    if str(REPO) not in sys.path:
        sys.path.insert(0, str(REPO))
    import oracle

    oracle.build()
    return oracle


def reduce_max(dist, v: float, device) -> float:
    """Max of `v` over the ranks of the default process group (identity
    without one). `device` holds the reduction tensor: the rank's GPU under
    NCCL, the CPU under gloo."""
    if not dist:
        return v
    import torch

    t = torch.tensor([float(v)], device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def measured_peak_gbs():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(workload: str):
    p = REPO / "profiles" / "traffic.json"
    if p.exists():
        d = json.loads(p.read_text())
        if workload in d:
            return d[workload]
    return None


# ---------------------------------------------------------------------------
# Clock sampling (NVML) during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    """Samples SM clock and throttle reasons with `nvidia-smi -lms` in a child
    process (a separate process cannot take the benchmark down with it)."""

    FIELDS = ("pci.bus_id,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int, period_ms: int = 50):
        self.samples = []
        self.ok = False
        self.proc = None
        try:
            import subprocess

            import torch

            if device_index < 0:
                raise RuntimeError("clock sampling disabled")
            props = torch.cuda.get_device_properties(device_index)
            bus = props.pci_bus_id
            if isinstance(bus, str):
                self.bus_tail = bus.upper()[-7:]  # "1B:00.0"
            else:  # integer bus / device numbers
                self.bus_tail = f"{int(bus):02X}:{int(getattr(props, 'pci_device_id', 0)):02X}.0"
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", str(period_ms)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.ok = True
        except Exception as e:  # noqa: BLE001
            self.err = str(e)

    def _run(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9 or not parts[0].upper().endswith(self.bus_tail):
                continue
            self.samples.append((time.perf_counter(), parts))

    def start(self):
        if self.ok:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()

    def stop(self):
        if self.ok:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:  # noqa: BLE001
                self.proc.kill()
            self.t.join(timeout=5)

    def summary(self, t0: float, t1: float):
        if not self.ok:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "note": getattr(self, "err", "")}
        inside = [s for s in self.samples if t0 <= s[0] <= t1]
        note = "sampled during the timed region"
        if len(inside) < 3:
            inside = self.samples
            note = "timed region shorter than the sampling period: warm-up and timed samples"

        def num(x):
            try:
                return float(x)
            except ValueError:
                return None

        mhz = [num(p[1]) for _, p in inside if num(p[1]) is not None]
        mx = [num(p[2]) for _, p in inside if num(p[2]) is not None]
        reasons = set()
        for _, p in inside:
            for name, v in zip(("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"), p[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(inside), "note": note}


# ---------------------------------------------------------------------------
# Shared timing harness
# ---------------------------------------------------------------------------
class Ctx:
    """Per-rank state shared by the workloads."""

    def __init__(self, args):
        import torch

        self.args = args
        self.torch = torch
        self.rank = int(os.environ.get("RANK", 0))
        self.world = int(os.environ.get("WORLD_SIZE", 1))
        self.local = int(os.environ.get("LOCAL_RANK", 0))
        torch.cuda.set_device(self.local)
        self.dev = f"cuda:{self.local}"
        self.dist = None
        if self.world > 1:
            import datetime

            import torch.distributed as dist

            os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", self.local))
            self.dist = dist
        self.bolt = load_package()
        self.eng = self.bolt.Engine(self.local, scratch_bytes=args.scratch_gb << 30)
        self.lib = self.eng._lib
        self.stream = torch.cuda.current_stream(self.local)

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def max_over_ranks(self, v: float) -> float:
        return reduce_max(self.dist, v, self.dev)

    def check(self, what: str):
        st = self.lib.bolt_ctx_sync_status(self.eng._ctx, self.stream.cuda_stream)
        if st != 0:
            raise RuntimeError(f"{what}: status {st}: {self.lib.bolt_ctx_last_error(self.eng._ctx).decode()}")

    def kernel_times(self, last: int):
        kt = (C.c_double * 4096)()
        nk = self.lib.bolt_ctx_kernel_times(self.eng._ctx, kt, 4096)
        return [kt[i] for i in range(nk)][-last:]

    def timed(self, step, steps: int, warmup: int, marks_per_step: int = 1):
        """Runs warmup + K async steps; returns (device ms, launches, kernel ms
        list of the timed steps' profiled kernels, clocks). marks_per_step:
        profiled kernels per step (the kernel list holds the last K of them)."""
        torch = self.torch
        sampler = ClockSampler(self.local) if not self.args.no_clocks else ClockSampler(-1)
        sampler.start()
        for _ in range(warmup):
            step()
        self.check("warm-up")
        self.kernel_times(4096)
        self.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        launches = 0
        t0 = time.perf_counter()
        e0.record(self.stream)
        for _ in range(steps):
            launches += step()
        e1.record(self.stream)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        self.barrier()
        ms = self.max_over_ranks(e0.elapsed_time(e1))
        self.check("timed region")
        kms = self.kernel_times(steps * marks_per_step)
        sampler.stop()
        return ms, launches, kms, sampler.summary(t0, t1)

    def time_e2e(self, step, steps: int) -> float:
        """Device time per call of `step` (host buffers in, host results out),
        after the warm-up calls that fill the pinned-memory caches."""
        torch = self.torch
        for _ in range(max(self.args.warmup, 3)):
            step()
        torch.cuda.synchronize()
        self.barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(self.stream)
        for _ in range(steps):
            step()
        f1.record(self.stream)
        torch.cuda.synchronize()
        return self.max_over_ranks(f0.elapsed_time(f1) / steps)


def base_line(c: Ctx, ms: float, rows_per_step: float, alg_bytes: float, kms, kernel: str, workload: str,
              config: dict, launches: int, clocks, dtype: str, unit: str = "rows/s"):
    a = c.args
    peak, peak_kind = measured_peak_gbs()
    kern_ms = statistics.mean(kms) if kms else None
    achieved = alg_bytes / (kern_ms * 1e-3) / 1e9 if kern_ms else None
    step_ms = ms / a.steps
    return {
        "metric": METRIC, "value": c.world * rows_per_step * a.steps / (ms * 1e-3), "unit": unit,
        "n_gpus": c.world, "steps": a.steps, "warmup": a.warmup, "ms_per_step": step_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
        "data": "synthetic (seeded splitmix64 generator; no dataset)",
        "config": dict(config, parallelism=f"replicas x{c.world}" if c.world > 1 else "1 GPU"),
        "hbm_gbs_step": alg_bytes / (step_ms * 1e-3) / 1e9,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak if achieved else None, "traffic": profiled_traffic(workload),
                     "kernel": kernel, "kernel_ms": kern_ms, "algorithmic_bytes_per_launch": alg_bytes,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"},
        "gpu_launches": launches,
        "clocks": clocks,
    }


# ---------------------------------------------------------------------------
# Workload: filtered two-key GROUP BY (default)
# ---------------------------------------------------------------------------
FILTERED_AGGS = [("sum", "vd"), ("avg", "vd"), ("count_star", None), ("min", "vi"), ("max", "vi")]
FILTERED_DT = {"a": "i32", "b": "i32", "f": "i32", "vd": "f64", "vi": "i64"}
FILTERED_BYTES = 4 + 4 + 4 + 8 + 8
FILTERED_WORKLOAD = ("filtered two-key GROUP BY: 100M rows, (a,b) int32 pairs of 10M Zipf(1.1) ranks, "
                     "WHERE f < 50, SUM/AVG(vd f64), COUNT(*), MIN/MAX(vi i64)")


def gen_filtered(n: int, device: str | None):
    dg = datagen()
    cdf = dg.zipf_cdf(10_000_000, 1.1)
    if device is not None:
        return dg.groupby_filtered(n, seed=2, ranks=dg.zipf_ranks_torch(cdf, 2, n, device))
    return dg.groupby_filtered(n, seed=2, cdf=cdf)


def tier_flags(c: Ctx) -> int:
    """GROUP BY flags for --tier: the library's choice, the shared-memory tier
    over a global hash table, or the hash-partitioned tier."""
    return {"auto": 0, "global": c.bolt.FLAG_NO_PART, "part": c.bolt.FLAG_FORCE_PART}[c.args.tier]


class PreparedCall:
    """A prepared GROUP BY run through bolt_groupby with BOLT_FLAG_ASYNC."""

    def __init__(self, c: Ctx, pq):
        self.c, self.pq = c, pq
        self.ng = c.torch.zeros(1, dtype=c.torch.int64, device=c.dev)
        pq.out.n_groups_dev = self.ng.data_ptr()
        self.flags = c.bolt.FLAG_ASYNC | c.bolt.FLAG_KERNEL_TIMES | tier_flags(c)

    def __call__(self):
        c = self.c
        st = c.lib.bolt_groupby(c.eng._ctx, C.byref(self.pq.desc), C.byref(self.pq.out), self.flags,
                                C.c_void_p(c.stream.cuda_stream))
        if st != 0:
            raise RuntimeError(f"bolt_groupby: {c.lib.bolt_ctx_last_error(c.eng._ctx).decode()}")
        return int(c.lib.bolt_ctx_last_launches(c.eng._ctx))


PART_KERNELS = ("gb_spill_kernel + gb_part_count_kernel + gb_part_scan_kernel + gb_part_scatter_kernel + "
                "gb_part_reduce_kernel (hash-partitioned tier)")


def agg_kernel_name(c: Ctx, rows: int, tuned: bool) -> str:
    """Which aggregation kernels the timed GROUP BY runs: the partitioned
    tier's five when --tier part or the tuning cache chooses it; else the
    streaming kernel when the tuning cache (or, untuned, the library's default
    for dense inputs of 256K rows and more) chooses it, else the register-tile
    kernel."""
    if c.args.tier == "part":
        return PART_KERNELS
    staged = rows >= (1 << 18)
    lean = "gb_lean_kernel (streaming kernel compiled for the query's layout; misses to the global hash table)"
    if tuned:
        import tempfile
        with tempfile.NamedTemporaryFile("r", suffix=".txt") as f:
            c.eng.save_tuning(f.name)
            lines = [ln.split() for ln in open(f.name) if ln.strip() and not ln.startswith("#")]
        if len(lines) == 1 and len(lines[0]) >= 8:
            staged = int(lines[0][6]) > 0
            if len(lines[0]) >= 9 and int(lines[0][8]) == 1 and c.args.tier == "auto":
                return PART_KERNELS
    return lean if staged else "gb_agg_kernel"


def cpu_rows_per_s_groupby(table_np: dict, dts: dict, group_by, aggs, where, n_sample: int, runs: int = 5):
    """Rows/s of the oracle's 1-thread GROUP BY on the first n_sample rows:
    the median of `runs` timed runs after one warm-up run."""
    orc = oracle_mod()
    host = {k: orc.HostCol(np.ascontiguousarray(v[:n_sample]), dts[k]) for k, v in table_np.items()}
    orc.groupby(host, group_by, aggs, where=where)
    times = []
    for _ in range(runs):
        t0 = time.perf_counter()
        orc.groupby(host, group_by, aggs, where=where)
        times.append(time.perf_counter() - t0)
    return n_sample / statistics.median(times)


def w_groupby_filtered(c: Ctx):
    a = c.args
    torch = c.torch
    progress(f"generating {a.rows} rows")
    data = gen_filtered(a.rows, c.dev)
    progress("pinning and uploading")
    host = {k: torch.from_numpy(v).pin_memory() for k, v in data.items()}
    dev = {k: c.bolt.Column(host[k].to(c.dev), FILTERED_DT[k]) for k in data}
    torch.cuda.synchronize()
    progress("prepared; timing")
    pq = c.eng.prepare_groupby(dev, ["a", "b"], FILTERED_AGGS, [("f", "<", 50)], groups_hint=a.groups_hint,
                               out_cap=max(2 * a.groups_hint, 1 << 20))
    tuned = None
    if a.tuning:
        c.eng.load_tuning(a.tuning)
        tuned = {"loaded": os.path.basename(a.tuning)}
    elif not a.no_tune:
        progress("autotuning")
        best = c.eng.autotune_groupby(pq)
        tuned = {"best_ms": best}
        progress(f"autotuned: {best:.3f} ms")
    if a.save_tuning:
        c.eng.save_tuning(a.save_tuning)
    kernel = agg_kernel_name(c, a.rows, tuned is not None)
    call = PreparedCall(c, pq)
    ms, launches, kms, clocks = c.timed(call, a.steps, a.warmup)
    n_groups = int(call.ng.item())
    progress(f"timed: {ms / a.steps:.3f} ms/step, {n_groups} groups")
    alg = a.rows * FILTERED_BYTES
    line = base_line(c, ms, a.rows, alg, kms, kernel, "groupby_filtered",
                     {"workload": FILTERED_WORKLOAD,
                      "rows": a.rows, "groups": n_groups, "groups_hint": a.groups_hint,
                      "autotuned": tuned,
                      "l2": "inputs (2.8 GB) larger than L2 (126 MB); no flush needed"},
                     launches, clocks, "int64/f64")
    if a.e2e_steps > 0:
        hcols = {k: c.bolt.Column(host[k], FILTERED_DT[k]) for k in data}
        res = {}

        def e2e():
            res["r"] = c.eng.execute_groupby(hcols, ["a", "b"], FILTERED_AGGS, where=[("f", "<", 50)],
                                             groups_hint=a.groups_hint)

        progress("end-to-end")
        e_ms = c.time_e2e(e2e, a.e2e_steps)
        line["e2e"] = {"value": c.world * a.rows / (e_ms * 1e-3), "unit": "rows/s", "h2d_bytes_per_step": alg,
                       "d2h_bytes_per_step": res["r"].n_groups * (4 + 4 + 8 * 5), "ms_per_step": e_ms,
                       "path": "Engine.execute_groupby on pinned host columns (H2D + GROUP BY + D2H)"}
    if c.world == 1 and not a.no_cpu:
        progress("CPU baseline")
        ns = min(a.cpu_rows, a.rows)
        rps = cpu_rows_per_s_groupby(data, FILTERED_DT, ["a", "b"], FILTERED_AGGS, [("f", "<", 50)], ns)
        line["cpu_baseline"] = {"value": rps, "unit": "rows/s", "cores": 1, "kind": "port",
                                "sample": f"first {ns} rows of the workload; CPU restatement of the reference's "
                                          "host GROUP BY (oracle), 1 thread; median of 5 runs after 1 warm-up"}
    return line


# ---------------------------------------------------------------------------
# Workload: plain single-key GROUP BY (1M rows)
# ---------------------------------------------------------------------------
PLAIN_AGGS = [("sum", "v"), ("count_star", None), ("min", "v"), ("max", "v")]
PLAIN_DT = {"k": "i32", "v": "i64"}


def w_groupby_plain(c: Ctx):
    a = c.args
    torch = c.torch
    n = a.plain_rows
    data = datagen().groupby_small(n, seed=1)
    host = {k: torch.from_numpy(v).pin_memory() for k, v in data.items()}
    dev = {k: c.bolt.Column(host[k].to(c.dev), PLAIN_DT[k]) for k in data}
    pq = c.eng.prepare_groupby(dev, ["k"], PLAIN_AGGS, groups_hint=1024)
    call = PreparedCall(c, pq)
    ms, launches, kms, clocks = c.timed(call, a.steps, a.warmup)
    alg = n * 12
    line = base_line(c, ms, n, alg, kms, agg_kernel_name(c, n, False), "groupby_plain",
                     {"workload": "plain single-key GROUP BY: 1M rows, k int32 U[0,1024), v int64 U[-1e6,1e6]; "
                                  "SUM, COUNT(*), MIN, MAX", "rows": n, "groups_hint": 1024,
                      "l2": "12 MB input fits in L2: warm-L2 figure (launch-bound workload)"},
                     launches, clocks, "int64")
    hcols = {k: c.bolt.Column(host[k], PLAIN_DT[k]) for k in data}
    e_ms = c.time_e2e(lambda: c.eng.execute_groupby(hcols, ["k"], PLAIN_AGGS, groups_hint=1024), a.e2e_steps or 3)
    line["e2e"] = {"value": n / (e_ms * 1e-3), "unit": "rows/s", "h2d_bytes_per_step": alg,
                   "d2h_bytes_per_step": 1024 * (4 + 32), "ms_per_step": e_ms}
    if not a.no_cpu:
        rps = cpu_rows_per_s_groupby(data, PLAIN_DT, ["k"], PLAIN_AGGS, [], n)
        line["cpu_baseline"] = {"value": rps, "unit": "rows/s", "cores": 1, "kind": "port",
                                "sample": f"all {n} rows, oracle GROUP BY, 1 thread"}
    return line


# ---------------------------------------------------------------------------
# Workload: hash join then aggregate
# ---------------------------------------------------------------------------
def w_join_groupby(c: Ctx):
    a = c.args
    torch = c.torch
    dg = datagen()
    nb, npr = a.build_rows, a.probe_rows
    bt = dg.join_build(nb, seed=3)
    pt = join_probe_host(dg, npr, nb)
    bk = c.bolt.Column(torch.from_numpy(bt["k"]).to(c.dev), "i64")
    bg = c.bolt.Column(torch.from_numpy(bt["g"]).to(c.dev), "i32")
    pk = c.bolt.Column(torch.from_numpy(pt["fk"]).to(c.dev), "i64")
    am = c.bolt.Column(torch.from_numpy(pt["amount"]).to(c.dev), "dec128", scale=2)
    abi = importlib.import_module("craton_bolt_b200._abi")
    g = torch.empty(4096, dtype=torch.int32, device=c.dev)
    s = torch.empty((4096, 2), dtype=torch.int64, device=c.dev)
    cnt = torch.empty(4096, dtype=torch.int64, device=c.dev)
    gm = abi.ColMut(g.data_ptr(), None, 4096, abi.I32, 0)
    sm = abi.ColMut(s.data_ptr(), None, 4096, abi.DEC128, 2)
    cm = abi.ColMut(cnt.data_ptr(), None, 4096, abi.I64, 0)
    ng = C.c_uint64(0)
    flags = c.bolt.FLAG_ASYNC | c.bolt.FLAG_KERNEL_TIMES
    bkv, bgv, pkv, amv = bk.view(), bg.view(), pk.view(), am.view()

    def step():
        t = C.c_void_p()
        st = c.lib.bolt_hash_join_build(c.eng._ctx, C.byref(bkv), C.byref(bgv), flags,
                                        C.c_void_p(c.stream.cuda_stream), C.byref(t))
        if st != 0:
            raise RuntimeError(c.lib.bolt_ctx_last_error(c.eng._ctx).decode())
        n_l = int(c.lib.bolt_ctx_last_launches(c.eng._ctx))
        st = c.lib.bolt_join_groupby(c.eng._ctx, t, C.byref(pkv), C.byref(amv), C.byref(gm), C.byref(sm),
                                     C.byref(cm), C.byref(ng), flags, C.c_void_p(c.stream.cuda_stream))
        if st != 0:
            raise RuntimeError(c.lib.bolt_ctx_last_error(c.eng._ctx).decode())
        n_l += int(c.lib.bolt_ctx_last_launches(c.eng._ctx))
        c.lib.bolt_hash_join_release(c.eng._ctx, t)
        return n_l

    ms, launches, kms, clocks = c.timed(step, a.steps, a.warmup, marks_per_step=2)
    # kernel times alternate build, probe-aggregate: the probe side dominates
    probe_k = kms[1::2] if len(kms) >= 2 else kms
    alg_probe = npr * 24
    alg = nb * 12 + npr * 24
    line = base_line(c, ms, npr, alg_probe, probe_k, "gb_agg_kernel (join lookup source)", "join_groupby",
                     {"workload": "hash inner join then aggregate: build 10M unique shuffled int64 keys + int32 g; "
                                  "probe 200M int64 fk (90% match), Decimal128(15,2) amount; GROUP BY g SUM, COUNT(*)",
                      "build_rows": nb, "probe_rows": npr, "algorithmic_bytes_step": alg,
                      "l2": "inputs (4.9 GB) larger than L2"}, launches, clocks, "int64/dec128")
    line["note"] = "value counts probe rows per second; one step = build + fused probe/aggregate"
    if not a.no_cpu:
        orc = oracle_mod()
        ns = min(a.cpu_rows, npr)
        t0 = time.perf_counter()
        orc.join_groupby(orc.HostCol(bt["k"], "i64"), bt["g"], orc.HostCol(pt["fk"][:ns], "i64"),
                         orc.HostCol(pt["amount"][:ns], "dec128", scale=2))
        line["cpu_baseline"] = {"value": ns / (time.perf_counter() - t0), "unit": "rows/s", "cores": 1,
                                "kind": "port", "sample": f"full build + first {ns} probe rows, oracle hash join "
                                                          "+ GROUP BY, 1 thread"}
    return line


def join_probe_host(dg, npr: int, nb: int) -> dict:
    """The probe side (fk, amount) generated in 32M-row chunks on every host
    thread (each chunk is a pure function of its row range)."""
    from concurrent.futures import ThreadPoolExecutor

    fk = np.empty(npr, np.int64)
    amount = np.empty((npr, 2), np.int64)

    def part(s):
        ch = dg.join_probe(min(1 << 25, npr - s), nb, seed=3, start=s)
        fk[s:s + len(ch["fk"])] = ch["fk"]
        amount[s:s + len(ch["fk"])] = ch["amount"]

    threads = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    with ThreadPoolExecutor(max_workers=threads) as pool:
        list(pool.map(part, range(0, npr, 1 << 25)))
    return {"fk": fk, "amount": amount}


# ---------------------------------------------------------------------------
# Workloads: ORDER BY radix sort
# ---------------------------------------------------------------------------
def w_sort(c: Ctx, kind: str):
    a = c.args
    torch = c.torch
    dg = datagen()
    if kind == "i64":
        n = a.sort_rows
        keys = np.empty(n, np.int64)
        dg._chunked(n, lambda a, b: keys.__setitem__(slice(a, b), dg.uniform_u64(4, 31, b - a, a).view(np.int64)))
        dt, kb, np_ = "i64", 8, 8
    else:
        n = a.sortf_rows
        keys = dg.sort_f32(n, seed=5)
        dt, kb, np_ = "f32", 4, 4
    col = c.bolt.Column(torch.from_numpy(keys).to(c.dev), dt)
    perm = torch.empty(n, dtype=torch.int32, device=c.dev)
    abi = importlib.import_module("craton_bolt_b200._abi")
    kv = col.view()
    pm = abi.ColMut(perm.data_ptr(), None, n, abi.U32, 0)
    flags = c.bolt.FLAG_ASYNC | c.bolt.FLAG_KERNEL_TIMES

    def step():
        st = c.lib.bolt_radix_sort_perm(c.eng._ctx, C.byref(kv), 0, 0, C.byref(pm), flags,
                                        C.c_void_p(c.stream.cuda_stream))
        if st != 0:
            raise RuntimeError(c.lib.bolt_ctx_last_error(c.eng._ctx).decode())
        return int(c.lib.bolt_ctx_last_launches(c.eng._ctx))

    ms, launches, kms, clocks = c.timed(step, a.steps, a.warmup)
    # pass accounting: histogram reads keys once; each 8-bit pass reads and
    # writes (key + u32 payload); the first pass reads only the key, the last
    # writes only the payload.
    passes = np_
    alg = n * (kb + kb + (passes - 2) * 2 * (kb + 4) + (kb + kb + 4) + (kb + 4 + 4))
    line = base_line(c, ms, n, alg, kms, "sort (histogram + passes)", f"sort_{kind}",
                     {"workload": f"ORDER BY radix sort: {n} {dt} keys" +
                                  (" uniform over the full range" if kind == "i64" else
                                   " incl. negatives, +-0, +-inf, 0.1% NaN"),
                      "rows": n, "passes": passes, "algorithmic_bytes": alg,
                      "minimum_bytes": n * (kb + 4), "l2": "inputs larger than L2"},
                     launches, clocks, dt)
    if not a.no_cpu:
        orc = oracle_mod()
        ns = min(a.cpu_rows, n)
        t0 = time.perf_counter()
        orc.sort_perm(orc.HostCol(keys[:ns], dt))
        line["cpu_baseline"] = {"value": ns / (time.perf_counter() - t0), "unit": "rows/s", "cores": 1,
                                "kind": "port", "sample": f"first {ns} keys, stable LSD sort in the oracle, 1 thread"}
    return line


# ---------------------------------------------------------------------------
# Workload: WHERE compaction
# ---------------------------------------------------------------------------
def w_compact(c: Ctx):
    a = c.args
    torch = c.torch
    data = gen_filtered(a.rows, c.dev)
    dev = {k: c.bolt.Column(torch.from_numpy(v).to(c.dev), FILTERED_DT[k]) for k, v in data.items()}
    abi = importlib.import_module("craton_bolt_b200._abi")
    names = list(dev)
    views = (abi.ColView * len(names))(*[dev[k].view() for k in names])
    outs = {k: torch.empty_like(dev[k].data) for k in names}
    muts = (abi.ColMut * len(names))(*[abi.ColMut(outs[k].data_ptr(), None, a.rows, abi.DTYPE_CODES[FILTERED_DT[k]], 0)
                                       for k in names])
    pred = (abi.Pred * 1)(abi.Pred(names.index("f"), abi.CMP_CODES["<"], 50, 0.0))
    nout = C.c_uint64(0)
    flags = c.bolt.FLAG_ASYNC | c.bolt.FLAG_KERNEL_TIMES

    def step():
        st = c.lib.bolt_compact(c.eng._ctx, views, len(names), pred, 1, muts, None, C.byref(nout), flags,
                                C.c_void_p(c.stream.cuda_stream))
        if st != 0:
            raise RuntimeError(c.lib.bolt_ctx_last_error(c.eng._ctx).decode())
        return int(c.lib.bolt_ctx_last_launches(c.eng._ctx))

    ms, launches, kms, clocks = c.timed(step, a.steps, a.warmup)
    alg = a.rows * FILTERED_BYTES * 1.5  # read all columns, write the ~50% kept
    kernel = ("compact_count_kernel + compact_scan_kernel + compact_bulk_kernel (two-pass form)"
              if a.rows >= (1 << 22) else "compact_bulk_kernel")
    line = base_line(c, ms, a.rows, alg, kms, kernel, "compact",
                     {"workload": "WHERE f < 50 compaction of 5 columns (28 B/row), 100M rows", "rows": a.rows,
                      "l2": "inputs larger than L2"}, launches, clocks, "mixed")
    if not a.no_cpu:
        orc = oracle_mod()
        ns = min(a.cpu_rows, a.rows)
        host = {k: orc.HostCol(np.ascontiguousarray(v[:ns]), FILTERED_DT[k]) for k, v in data.items()}
        orc.compact(host, where=[("f", "<", 50)])
        times = []
        for _ in range(5):
            t0 = time.perf_counter()
            orc.compact(host, where=[("f", "<", 50)])
            times.append(time.perf_counter() - t0)
        line["cpu_baseline"] = {"value": ns / statistics.median(times), "unit": "rows/s", "cores": 1, "kind": "port",
                                "sample": f"first {ns} rows, the oracle's order-preserving filter (selected row "
                                          "indices), 1 thread; median of 5 runs after 1 warm-up"}
    return line


# ---------------------------------------------------------------------------
# Workload: batched / served stream of filter + GROUP BY queries
# ---------------------------------------------------------------------------
CARDS = [10, 32, 100, 316, 1000, 3162, 10_000, 31_623, 100_000, 316_228, 1_000_000]


def batch_queries(n_q: int, table_rows: int, seed: int = 7, max_rows: float = 5e7):
    rng = np.random.default_rng(seed)
    qs = []
    for i in range(n_q):
        rows = int(math.exp(rng.uniform(math.log(1e4), math.log(min(max_rows, table_rows)))))
        begin = int(rng.integers(0, table_rows - rows + 1))
        card = CARDS[int(rng.integers(0, len(CARDS)))]
        qs.append({"begin": begin, "end": begin + rows, "card": card, "key": "k32" if i % 2 == 0 else "k64",
                   "val": "vi" if (i // 2) % 2 == 0 else "vd", "t": int(rng.integers(10, 100))})
    return qs


def w_batch(c: Ctx):
    a = c.args
    torch = c.torch
    dg = datagen()
    n = a.batch_table_rows
    base = {"k32": (dg.uniform_u64(8, 1, n) >> np.uint64(33)).astype(np.int64),
            "vi": (dg.uniform_u64(8, 2, n) % np.uint64(2_000_001)).astype(np.int64) - 1_000_000,
            "vd": dg.normal_f64(8, 3, n, 1e3),
            "f": ((dg.uniform_u64(8, 4, n) >> np.uint64(32)) % np.uint64(100)).astype(np.int32)}
    dev = {"vi": c.bolt.Column(torch.from_numpy(base["vi"]).to(c.dev), "i64"),
           "vd": c.bolt.Column(torch.from_numpy(base["vd"]).to(c.dev), "f64"),
           "f": c.bolt.Column(torch.from_numpy(base["f"]).to(c.dev), "i32")}
    for card in CARDS:
        kk = base["k32"] % card
        dev[f"k32_{card}"] = c.bolt.Column(torch.from_numpy(kk.astype(np.int32)).to(c.dev), "i32")
        dev[f"k64_{card}"] = c.bolt.Column(torch.from_numpy(kk * 1_000_003 - (1 << 40)).to(c.dev), "i64")

    def prep(q, sliced=False):
        """A query's descriptor: a row range of the resident columns (batched
        and served paths), or, for the one-at-a-time bolt_groupby path whose
        descriptor has no row range, column views of exactly its rows."""
        kname = f"{q['key']}_{q['card']}"
        t = {kname: dev[kname], q["val"]: dev[q["val"]], "f": dev["f"]}
        aggs, where = [("sum", q["val"]), ("count_star", None)], [("f", "<", q["t"])]
        if sliced:
            t = {k: c.bolt.Column(v.data[q["begin"]:q["end"]], v.dtype) for k, v in t.items()}
            return c.eng.prepare_groupby(t, [kname], aggs, where, groups_hint=q["card"])
        return c.eng.prepare_groupby(t, [kname], aggs, where, groups_hint=q["card"], rows=(q["begin"], q["end"]))

    def measure(qs):
        """One-at-a-time bolt_groupby launches vs the continuous-batching
        server on the same queries: throughput, equality, Poisson latency."""
        total_rows = sum(q["end"] - q["begin"] for q in qs)
        prepared = [prep(q, sliced=True) for q in qs]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        lat_single = []
        for pq in prepared:
            s0 = time.perf_counter()
            st = c.lib.bolt_groupby(c.eng._ctx, C.byref(pq.desc), C.byref(pq.out), 0,
                                    C.c_void_p(c.stream.cuda_stream))
            if st != 0:
                raise RuntimeError(c.lib.bolt_ctx_last_error(c.eng._ctx).decode())
            lat_single.append((time.perf_counter() - s0) * 1e6)
        single_s = time.perf_counter() - t0
        single_groups = [int(pq.out.n_groups) for pq in prepared]
        single_qps = len(qs) / single_s
        del prepared
        scratch = min(a.server_scratch_gb << 30, int(torch.cuda.mem_get_info()[0] * 0.8))
        srv = c.bolt.Server(c.local, scratch_bytes=scratch, max_batch=a.max_batch, n_lanes=a.lanes)
        try:
            prepared2 = [prep(q) for q in qs]
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            tickets = srv.submit_many(prepared2)  # the whole burst in one call
            for t in tickets:
                srv.wait(t)
            batch_s = time.perf_counter() - t0
            batch_qps = len(qs) / batch_s
            same = all(int(p2.out.n_groups) == g for p2, g in zip(prepared2, single_groups))
            del prepared2
            # Poisson arrivals at 80% of the one-at-a-time capacity: p50 / p99.
            rate = 0.8 * single_qps
            rng = np.random.default_rng(11)
            gaps = rng.exponential(1.0 / rate, len(qs))
            prepared3 = [prep(q) for q in qs]
            torch.cuda.synchronize()
            tickets = []
            # No collector pause inside the arrival loop: a full collection over
            # the prepared queries stalls the submitter for tens of
            # milliseconds, which then submits the overdue arrivals at once.
            gc.collect()
            gc.disable()
            try:
                t0 = time.perf_counter()
                nxt = t0
                for pq, gap in zip(prepared3, gaps):
                    nxt += gap
                    while time.perf_counter() < nxt:
                        pass
                    tickets.append(srv.submit(pq))
                lat_poisson = [srv.wait(t)[1] for t in tickets]
            finally:
                gc.enable()
        finally:
            srv.close()
        # The same Poisson arrivals served one query at a time (FIFO): latency
        # from arrival to completion.
        prepared4 = [prep(q, sliced=True) for q in qs]
        torch.cuda.synchronize()
        lat_single_poisson = []
        gc.collect()
        gc.disable()
        try:
            t0 = time.perf_counter()
            arrive = t0
            for pq, gap in zip(prepared4, gaps):
                arrive += gap
                while time.perf_counter() < arrive:
                    pass
                st = c.lib.bolt_groupby(c.eng._ctx, C.byref(pq.desc), C.byref(pq.out), 0,
                                        C.c_void_p(c.stream.cuda_stream))
                if st != 0:
                    raise RuntimeError(c.lib.bolt_ctx_last_error(c.eng._ctx).decode())
                lat_single_poisson.append((time.perf_counter() - arrive) * 1e6)
        finally:
            gc.enable()
        del prepared4
        return {"queries": len(qs), "rows_total": total_rows, "batched_qps": batch_qps,
                "one_at_a_time_qps": single_qps, "speedup": batch_qps / single_qps,
                "rows_per_s_batched": total_rows / batch_s, "batch_s": batch_s,
                "results_equal_alone_vs_mix": same,
                "latency_us": {"one_at_a_time_p50": float(np.percentile(lat_single, 50)),
                               "one_at_a_time_p99": float(np.percentile(lat_single, 99)),
                               "served_poisson_p50": float(np.percentile(lat_poisson, 50)),
                               "served_poisson_p99": float(np.percentile(lat_poisson, 99)),
                               "one_at_a_time_poisson_p50": float(np.percentile(lat_single_poisson, 50)),
                               "one_at_a_time_poisson_p99": float(np.percentile(lat_single_poisson, 99)),
                               "poisson_rate_qps": rate}}

    main_mix = measure(batch_queries(a.batch_queries, n))
    # The same stream with rows per query log-uniform 10K..1M: launch-bound
    # queries, where batching is what pays.
    small_mix = measure(batch_queries(a.batch_queries, n, seed=8, max_rows=1e6))
    line = {
        "metric": METRIC, "value": main_mix["batched_qps"], "unit": "queries/s", "n_gpus": c.world, "steps": 1,
        "warmup": 0, "ms_per_step": main_mix["batch_s"] * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32/int64/f64", "data": "synthetic (seeded)",
        "config": {"workload": f"{a.batch_queries} filter + GROUP BY queries over resident {n}-row columns, "
                               "rows/query log-uniform 1e4..5e7, cardinality log-uniform 10..1e6, int32/int64 keys, "
                               "int64/f64 values", "lanes": a.lanes, "max_batch": a.max_batch},
        **main_mix,
        "small_query_mix": dict(small_mix, workload="same, rows/query log-uniform 1e4..1e6"),
        "gpu_launches": None,
    }
    return line


WORKLOADS = {"groupby_filtered": w_groupby_filtered, "groupby_plain": w_groupby_plain,
             "join_groupby": w_join_groupby, "sort_i64": lambda c: w_sort(c, "i64"),
             "sort_f32": lambda c: w_sort(c, "f32"), "compact": w_compact, "batch": w_batch}


# ---------------------------------------------------------------------------
# Every other operator, summarised inside the default line
# ---------------------------------------------------------------------------
OPERATORS = ["groupby_plain", "join_groupby", "sort_i64", "sort_f32", "compact", "batch"]
OP_KEYS = ("value", "unit", "ms_per_step", "steps", "warmup", "dtype", "config", "roofline", "cpu_baseline", "e2e",
           "gpu_launches", "clocks", "note", "batched_qps", "one_at_a_time_qps", "speedup", "latency_us",
           "results_equal_alone_vs_mix", "rows_per_s_batched")


def run_operators(c: Ctx) -> dict:
    """Each other workload at its own full size with fewer repeats (at most 5
    timed steps after 3 warm-up steps, one end-to-end step), summarised as a
    sub-line of the default line's `operators` map."""
    import copy

    import torch

    saved = c.args
    out = {}
    for name in OPERATORS:
        a = copy.copy(saved)
        a.steps, a.warmup, a.e2e_steps = min(saved.steps, 5), 3, 1
        c.args = a
        progress(f"operator {name}")
        try:
            line = WORKLOADS[name](c)
            d = {k: line[k] for k in OP_KEYS if k in line}
            if "small_query_mix" in line:
                sm = line["small_query_mix"]
                d["small_query_mix"] = {k: sm[k] for k in ("batched_qps", "one_at_a_time_qps", "speedup", "latency_us",
                                                           "results_equal_alone_vs_mix", "workload") if k in sm}
            out[name] = d
        except Exception as e:  # noqa: BLE001  (one failing operator must not hide the others)
            out[name] = {"error": f"{type(e).__name__}: {e}"[:400]}
        finally:
            c.args = saved
            torch.cuda.synchronize()
            torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------------------
# Reference arm
# ---------------------------------------------------------------------------
def run_reference(args):
    """The reference's host GROUP BY path (restated in C: the reference is
    Rust and cannot be built here) over the full workload, every step, on
    every host thread: rows are range-partitioned by key and each partition
    is folded in row order by one thread, so the result equals the
    sequential fold's. Partitioning, folding, the per-partition sort and the
    output assembly are all timed."""
    progress(f"reference arm: generating {args.rows} rows on the host")
    data = gen_filtered(args.rows, None)
    orc = oracle_mod()
    host = {k: orc.HostCol(np.ascontiguousarray(v), FILTERED_DT[k]) for k, v in data.items()}
    threads = orc.host_threads()
    times, groups = [], None
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        r = orc.groupby(host, ["a", "b"], FILTERED_AGGS, where=[("f", "<", 50)], threads=threads)
        dt = time.perf_counter() - t0
        groups = r["n_groups"]
        del r
        if i >= args.warmup:
            times.append(dt)
        progress(f"reference step {i}: {dt * 1e3:.1f} ms")
    total = sum(times)
    value = args.rows * len(times) / total
    line = {"metric": METRIC, "value": value, "unit": "rows/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times),
            "ms_per_step_median": 1e3 * statistics.median(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64/f64",
            "data": "synthetic (seeded splitmix64 generator; same rows as the GPU arm)",
            "config": {"workload": FILTERED_WORKLOAD, "rows": args.rows, "groups": groups,
                       "rows_per_step": args.rows, "parallelism": f"host, {threads} threads"},
            "cpu_baseline": {"value": value, "unit": "rows/s", "cores": threads, "kind": "port",
                             "sample": f"all {args.rows} rows of the workload every step; the reference's host "
                                       "GROUP BY (HashMap fold in row order, sorted output) restated in C, on "
                                       f"{threads} threads (key-range partitions), everything timed"},
            "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="groupby_filtered", choices=sorted(WORKLOADS))
    ap.add_argument("--rows", type=int, default=100_000_000)
    ap.add_argument("--groups-hint", type=int, default=4_000_000)
    ap.add_argument("--plain-rows", type=int, default=1_000_000)
    ap.add_argument("--build-rows", type=int, default=10_000_000)
    ap.add_argument("--probe-rows", type=int, default=200_000_000)
    ap.add_argument("--sort-rows", type=int, default=256 << 20)
    ap.add_argument("--sortf-rows", type=int, default=64 << 20)
    ap.add_argument("--batch-queries", type=int, default=4096)
    ap.add_argument("--batch-table-rows", type=int, default=50_000_000)
    ap.add_argument("--max-batch", type=int, default=512)
    ap.add_argument("--lanes", type=int, default=4)
    ap.add_argument("--server-scratch-gb", type=int, default=64)
    ap.add_argument("--scratch-gb", type=int, default=16)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-rows", type=int, default=10_000_000)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-clocks", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="skip the GROUP BY autotuner")
    ap.add_argument("--tuning", default=None, help="load GROUP BY launch choices from this file instead of tuning")
    ap.add_argument("--save-tuning", default=None, help="write the GROUP BY launch choices to this file")
    ap.add_argument("--no-operators", action="store_true",
                    help="default workload: skip the other operators' summary lines (the `operators` map)")
    ap.add_argument("--tier", default="auto", choices=["auto", "global", "part"],
                    help="GROUP BY tier: the library's choice, shared-memory + global hash table, hash-partitioned")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", 0))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return
    progress(f"workload {args.workload}")
    c = Ctx(args)
    progress("context ready")
    line = WORKLOADS[args.workload](c)
    if args.workload == "groupby_filtered" and c.world == 1 and not args.no_operators:
        line["operators"] = run_operators(c)
    if c.rank == 0:
        print(json.dumps(line), flush=True)
    c.eng.close()
    if c.dist:
        c.dist.barrier()
        c.dist.destroy_process_group()


if __name__ == "__main__":
    main()
