#!/usr/bin/env python
"""Benchmark of the B200 relational hot path (one JSON line on rank 0).

Default workload: the filtered high-cardinality two-key GROUP BY
  SELECT a, b, SUM(vd), AVG(vd), COUNT(*), MIN(vi), MAX(vi)
  FROM t WHERE f < 50 GROUP BY a, b
over 100,000,000 seeded synthetic rows ((a, b) int32 pairs of 10M Zipf(1.1)
ranks, f int32 U[0,100), vd f64 N(0,1e3), vi int64 uniform).

  value      rows/s with the columns resident in HBM (device-timed, K steps)
  e2e        rows/s through the public API from pinned host columns,
             host->device copies and result readback inside the timed region
  roofline   the aggregation kernel's algorithmic bytes / its CUDA-event time
  cpu_baseline  the CPU oracle (restatement of the reference's host path)
             on a bounded sample of the same rows

`--impl reference` times the CPU restatement of the reference's host path
(the reference itself is Rust and cannot be built here) on the same
workload and prints the same line with "impl": "reference".
Multi-GPU (torchrun): independent replicas, one per rank; value sums all
ranks' rows over the max per-rank device time.
"""

from __future__ import annotations

import argparse
import importlib
import importlib.util
import json
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
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
    def __init__(self, device_index: int, period_s: float = 0.005):
        self.samples = []
        self.period = period_s
        self._stop = threading.Event()
        self.ok = False
        try:
            import pynvml
            import torch

            pynvml.nvmlInit()
            bus = torch.cuda.get_device_properties(device_index).pci_bus_id
            self.h = pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode() if isinstance(bus, str) else bus)
            self.nv = pynvml
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception as e:  # noqa: BLE001
            self.err = str(e)

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                mhz = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                rs = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                self.samples.append((time.perf_counter(), mhz, rs))
            except Exception:  # noqa: BLE001
                pass
            time.sleep(self.period)

    def start(self):
        if self.ok:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()

    def stop(self):
        if self.ok:
            self._stop.set()
            self.t.join()

    def summary(self, t0: float, t1: float):
        if not self.ok:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "note": getattr(self, "err", "")}
        inside = [s for s in self.samples if t0 <= s[0] <= t1]
        note = "sampled during the timed region"
        if len(inside) < 3:
            inside = self.samples
            note = "timed region shorter than the sampling period: warm-up and timed samples"
        nv = self.nv
        names = {
            "gpu_idle": getattr(nv, "nvmlClocksEventReasonGpuIdle", 0x1),
            "applications_clocks_setting": getattr(nv, "nvmlClocksEventReasonApplicationsClocksSetting", 0x2),
            "sw_power_cap": getattr(nv, "nvmlClocksEventReasonSwPowerCap", 0x4),
            "hw_slowdown": getattr(nv, "nvmlClocksEventReasonHwSlowdown", 0x8),
            "sync_boost": getattr(nv, "nvmlClocksEventReasonSyncBoost", 0x10),
            "sw_thermal_slowdown": getattr(nv, "nvmlClocksEventReasonSwThermalSlowdown", 0x20),
            "hw_thermal_slowdown": getattr(nv, "nvmlClocksEventReasonHwThermalSlowdown", 0x40),
            "hw_power_brake_slowdown": getattr(nv, "nvmlClocksEventReasonHwPowerBrakeSlowdown", 0x80),
        }
        reasons = set()
        for _, _, rs in inside:
            for k, bit in names.items():
                if rs & bit and k != "gpu_idle":
                    reasons.add(k)
        mhz = [s[1] for s in inside]
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(reasons), "samples": len(inside), "note": note}


# ---------------------------------------------------------------------------
# Workload: filtered two-key GROUP BY
# ---------------------------------------------------------------------------
FILTERED_AGGS = [("sum", "vd"), ("avg", "vd"), ("count_star", None), ("min", "vi"), ("max", "vi")]
FILTERED_DT = {"a": "i32", "b": "i32", "f": "i32", "vd": "f64", "vi": "i64"}
BYTES_PER_ROW = 4 + 4 + 4 + 8 + 8


def gen_filtered(n: int, device: str | None):
    load_package()
    dg = importlib.import_module("craton_bolt_b200.datagen")
    cdf = dg.zipf_cdf(10_000_000, 1.1)
    if device is not None:
        ranks = dg.zipf_ranks_torch(cdf, 2, n, device)
    else:
        ranks = dg.zipf_ranks(cdf, dg.unit_f64(dg.uniform_u64(2, 10, n)))
    return dg.groupby_filtered(n, seed=2, ranks=ranks)


class GroupbyCall:
    """Prebuilt C-ABI call of the filtered GROUP BY on device-resident columns."""

    def __init__(self, bolt, eng, dev_cols: dict, groups_hint: int, out_cap: int):
        import ctypes as C
        import torch

        abi = importlib.import_module("craton_bolt_b200._abi")
        self.C, self.abi, self.eng, self.lib = C, abi, eng, bolt.lib()
        names = list(dev_cols)
        self.keep = [dev_cols]
        self.views = (abi.ColView * len(names))(*[dev_cols[k].view() for k in names])
        self.kidx = (C.c_int32 * 2)(names.index("a"), names.index("b"))
        self.preds = (abi.Pred * 1)(abi.Pred(names.index("f"), abi.CMP_CODES["<"], 50, 0.0))
        self.specs = (abi.AggSpec * len(FILTERED_AGGS))(
            *[abi.AggSpec(abi.AGG_CODES[op], names.index(c) if c else -1) for op, c in FILTERED_AGGS])
        self.desc = abi.GroupbyDesc(self.views, len(names), self.kidx, 2, self.preds, 1, self.specs,
                                    len(FILTERED_AGGS), groups_hint)
        dev = dev_cols["a"].data.device
        self.outs = [torch.empty(out_cap, dtype=torch.int32, device=dev), torch.empty(out_cap, dtype=torch.int32, device=dev)]
        self.aouts = [torch.empty(out_cap, dtype=t, device=dev) for t in
                      (torch.float64, torch.float64, torch.int64, torch.int64, torch.int64)]
        self.ng = torch.zeros(1, dtype=torch.int64, device=dev)
        kd = [abi.I32, abi.I32]
        ad = [abi.F64, abi.F64, abi.I64, abi.I64, abi.I64]
        self.kmut = (abi.ColMut * 2)(*[abi.ColMut(t.data_ptr(), None, out_cap, d, 0) for t, d in zip(self.outs, kd)])
        self.amut = (abi.ColMut * 5)(*[abi.ColMut(t.data_ptr(), None, out_cap, d, 0) for t, d in zip(self.aouts, ad)])
        self.out = abi.GroupbyOut(self.kmut, self.amut, 0, self.ng.data_ptr())

    def __call__(self, stream_handle: int, flags: int):
        st = self.lib.bolt_groupby(self.eng._ctx, self.C.byref(self.desc), self.C.byref(self.out), flags,
                                   self.C.c_void_p(stream_handle))
        if st != 0:
            raise RuntimeError(f"bolt_groupby failed: {self.lib.bolt_ctx_last_error(self.eng._ctx).decode()}")
        return int(self.lib.bolt_ctx_last_launches(self.eng._ctx))


def cpu_sample_rows_per_s(data: dict, n_sample: int, threads: int = 1):
    sys.path.insert(0, str(REPO))
    import oracle

    oracle.build()
    oracle.lib().orc_set_threads(threads)
    host = {k: oracle.HostCol(np.ascontiguousarray(v[:n_sample]), FILTERED_DT[k]) for k, v in data.items()}
    t0 = time.perf_counter()
    oracle.groupby(host, ["a", "b"], FILTERED_AGGS, where=[("f", "<", 50)])
    dt = time.perf_counter() - t0
    return n_sample / dt, dt


def run_reference(args):
    """CPU restatement of the reference's host GROUP BY path, timed per step
    on a bounded sample of the workload's rows."""
    n_sample = args.reference_rows
    data = gen_filtered(n_sample, None)
    times = []
    for i in range(args.warmup + args.steps):
        rps, dt = cpu_sample_rows_per_s(data, n_sample)
        if i >= args.warmup:
            times.append(dt)
    total = sum(times)
    value = n_sample * len(times) / total
    line = {"metric": METRIC, "value": value, "unit": "rows/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64/f64",
            "data": "synthetic (seeded, same generator as the GPU arm)",
            "config": {"workload": "filtered two-key GROUP BY (Zipf(1.1) pairs, f < 50)", "rows_per_step": n_sample,
                       "rows_full": args.rows, "parallelism": "host"},
            "cpu_baseline": {"value": value, "unit": "rows/s", "cores": 1, "kind": "port",
                             "sample": f"first {n_sample} rows of the workload per step; the reference is Rust "
                                       "(no cargo here), timed as its C restatement, single-threaded as its "
                                       "host HashMap path"},
            "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--rows", type=int, default=100_000_000)
    ap.add_argument("--groups-hint", type=int, default=4_000_000)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-rows", type=int, default=10_000_000)
    ap.add_argument("--reference-rows", type=int, default=2_000_000)
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return

    import torch

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=torch.device("cuda", local))
    bolt = load_package()
    dev = f"cuda:{local}"
    data = gen_filtered(args.rows, dev)
    host = {k: torch.from_numpy(v).pin_memory() for k, v in data.items()}
    dev_cols = {k: bolt.Column(host[k].to(dev), FILTERED_DT[k]) for k in data}
    torch.cuda.synchronize()
    eng = bolt.Engine(local, scratch_bytes=8 << 30)
    call = GroupbyCall(bolt, eng, dev_cols, args.groups_hint, out_cap=max(2 * args.groups_hint, 1 << 20))
    s = torch.cuda.current_stream(local)
    flags = bolt.FLAG_ASYNC | bolt.FLAG_PROFILE

    sampler = ClockSampler(local)
    sampler.start()
    for _ in range(args.warmup):
        call(s.cuda_stream, flags)
    st = eng._lib.bolt_ctx_sync_status(eng._ctx, s.cuda_stream)
    if st != 0:
        raise RuntimeError(f"warm-up status {st}: {eng._lib.bolt_ctx_last_error(eng._ctx).decode()}")
    eng._lib.bolt_ctx_kernel_times(eng._ctx, None, 1 << 20)

    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches = 0
    t_wall0 = time.perf_counter()
    e0.record(s)
    for _ in range(args.steps):
        launches += call(s.cuda_stream, flags)
    e1.record(s)
    torch.cuda.synchronize()
    t_wall1 = time.perf_counter()
    if dist:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    st = eng._lib.bolt_ctx_sync_status(eng._ctx, s.cuda_stream)
    if st != 0:
        raise RuntimeError(f"timed-region status {st}: {eng._lib.bolt_ctx_last_error(eng._ctx).decode()}")
    import ctypes as C

    kt = (C.c_double * 4096)()
    nk = eng._lib.bolt_ctx_kernel_times(eng._ctx, kt, 4096)
    kms = [kt[i] for i in range(nk)][-args.steps:]
    sampler.stop()
    clocks = sampler.summary(t_wall0, t_wall1)
    n_groups = int(call.ng.item())

    if dist:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())

    # End to end through the public API: pinned host columns in, host result out.
    e2e_ms = None
    h2d = args.rows * BYTES_PER_ROW
    d2h = 0
    if args.e2e_steps > 0:
        host_cols = {k: bolt.Column(host[k], FILTERED_DT[k]) for k in data}
        eng.execute_groupby(host_cols, ["a", "b"], FILTERED_AGGS, where=[("f", "<", 50)],
                            groups_hint=args.groups_hint)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        f0.record(s)
        for _ in range(args.e2e_steps):
            r = eng.execute_groupby(host_cols, ["a", "b"], FILTERED_AGGS, where=[("f", "<", 50)],
                                    groups_hint=args.groups_hint)
        f1.record(s)
        torch.cuda.synchronize()
        e2e_ms = f0.elapsed_time(f1) / args.e2e_steps
        d2h = r.n_groups * (4 + 4 + 8 * 5)
        if dist:
            t = torch.tensor([e2e_ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            e2e_ms = float(t.item())

    if rank == 0:
        peak, peak_kind = measured_peak_gbs()
        alg_bytes = args.rows * BYTES_PER_ROW
        kern_ms = statistics.mean(kms) if kms else None
        achieved = alg_bytes / (kern_ms * 1e-3) / 1e9 if kern_ms else None
        step_ms = ms / args.steps
        line = {
            "metric": METRIC, "value": world * args.rows * args.steps / (ms * 1e-3), "unit": "rows/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64/f64",
            "data": "synthetic (seeded splitmix64 generator; no dataset)",
            "config": {"workload": "filtered two-key GROUP BY: 100M rows, (a,b) int32 pairs of 10M Zipf(1.1) "
                                   "ranks, WHERE f < 50, SUM/AVG(vd f64), COUNT(*), MIN/MAX(vi i64)",
                       "rows": args.rows, "groups": n_groups, "groups_hint": args.groups_hint,
                       "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
                       "l2": "inputs (2.8 GB) larger than L2 (126 MB); no flush needed"},
            "hbm_gbs_step": alg_bytes / (step_ms * 1e-3) / 1e9,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak if achieved else None, "traffic": profiled_traffic("groupby_filtered"),
                         "kernel": "gb_agg_kernel", "kernel_ms": kern_ms,
                         "algorithmic_bytes_per_launch": alg_bytes, "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"},
            "gpu_launches": launches,
            "clocks": clocks,
            "e2e": {"value": (world * args.rows / (e2e_ms * 1e-3)) if e2e_ms else None, "unit": "rows/s",
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms,
                    "path": "Engine.execute_groupby on pinned host columns (H2D + GROUP BY + D2H)"},
        }
        if world == 1 and not args.no_cpu:
            rps, _ = cpu_sample_rows_per_s(data, min(args.cpu_rows, args.rows))
            line["cpu_baseline"] = {"value": rps, "unit": "rows/s", "cores": 1, "kind": "port",
                                    "sample": f"first {min(args.cpu_rows, args.rows)} rows of the workload, CPU "
                                              "restatement of the reference's host GROUP BY (oracle), 1 thread"}
        print(json.dumps(line), flush=True)
    eng.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
