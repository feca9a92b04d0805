"""Benchmark of the filter -> group_by -> fused-aggregate path on B200.

Default workload ("hash"): 100M rows; key int32 Zipf(s=1.1) over 1M values; v1, v2 float64
N(0,1); v3 int64 U[0,1e9); 5% nulls on v1, v2, v3; filter (v1 > -0.5) & (v3 % 7 != 0);
aggregates sum/mean(v1), min/max(v2), sum(v3), len. Seeded synthetic data, generated on the GPU
and excluded from timing. Inputs are 2.84 GB (> 126 MB L2), so no L2 flush is needed.

One step = one full pmb_groupby call on device-resident inputs (sketch, table init, fused hash
aggregation, finalize, group-count readback). `value` = rows of all ranks / max step time;
`e2e` = the same call with inputs in pinned host memory and results copied back to the host.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload hash|small|sort|batch]

Every line of the default workload also carries "batched": the batched workload (4096 independent
filter -> group_by queries, ~500M rows in total) run through pmb_groupby_batched with the learned
strategy selector, against the same queries run one by one through pmb_groupby with the plain
cardinality heuristic (total rows/s of both). --workload batch makes that the headline line.

--impl reference times the CPU restatement of the reference's algorithm (the oracle, all host
threads) on a bounded sample of the same workload; the reference itself (Rust + Metal) cannot
run on this machine.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "polars-metal_b200"))
sys.path.insert(0, str(ROOT))

METRIC = "rows/s filter→group_by→agg @100M rows, % of HBM roofline; batched+learned vs plain"

WORKLOADS = {
    "hash": ("make_hash", 100_000_000,
             "hash: 100M rows, int32 Zipf(1.1) keys over 1M values, f64 v1/v2 N(0,1), i64 v3 U[0,1e9), 5% nulls, "
             "filter (v1>-0.5)&(v3%7!=0), sum/mean(v1) min/max(v2) sum(v3) len"),
    "small": ("make_small", 1_000_000,
              "small: 1M rows, int64 key U[0,1000), f64 v1 N(0,1), i64 v2 U[-1e6,1e6], 1% nulls, filter v1>0, "
              "sum/mean(v1) min/max(v2) len"),
    "sort": ("make_sort", 200_000_000,
             "sort: 200M rows, (int64 from 781,250 values in [0,2^40), int32 U[0,64)) keys ~50M groups, f32 v U(0,1), "
             "i64 vi, sum/min/max/len"),
}


BATCH_QUERIES, BATCH_ROWS = 4096, 500_000_000
BATCH_DESC = ("batch: 4096 independent queries, rows lognormal(ln 1e5, 1.5) clipped to [1K, 10M] and scaled to 500M "
              "in total; key int32, cardinality log-uniform [10, 1e6] (at most the rows), Zipf s ~ U[0, 1.5]; "
              "v f64 N(0,1) with 1% nulls; filter v > -1; sum/mean/min/max(v), len")


def load_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        try:
            return float(json.loads(p.read_text())["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


class ClockSampler:
    """Samples SM clocks and throttle reasons while the timed region runs: NVML queries (read only)
    when the region starts, every 2 ms in a thread, and when it ends; or nvidia-smi every 50 ms when
    NVML is not importable."""

    REASONS = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40, "sw_power_cap": 0x4}

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.samples = []  # (sm_mhz, max_mhz, reasons)
        self._stop = threading.Event()
        self._proc = None
        self._t = None

    def __enter__(self):
        try:
            import pynvml

            pynvml.nvmlInit()
            dev = pynvml.nvmlDeviceGetHandleByIndex(self.gpu)
            mx = pynvml.nvmlDeviceGetMaxClockInfo(dev, pynvml.NVML_CLOCK_SM)
            reasons_of = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                pynvml.nvmlDeviceGetCurrentClocksThrottleReasons

            def sample():
                try:
                    sm = pynvml.nvmlDeviceGetClockInfo(dev, pynvml.NVML_CLOCK_SM)
                    bits = reasons_of(dev)
                    self.samples.append((float(sm), float(mx), {n for n, m in self.REASONS.items() if bits & m}))
                except Exception:
                    pass

            def loop():
                while not self._stop.wait(0.002):
                    sample()
                sample()

            sample()
            self._t = threading.Thread(target=loop, daemon=True)
            self._t.start()
            return self
        except Exception:
            pass
        try:
            fields = ("clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                      "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
            self._proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={fields}", "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)

            def read():
                names = ["hw_slowdown", "sw_thermal_slowdown", "hw_thermal_slowdown", "sw_power_cap"]
                for line in self._proc.stdout:
                    f = [x.strip() for x in line.split(",")]
                    try:
                        self.samples.append((float(f[0]), float(f[1]),
                                             {n for n, v in zip(names, f[2:6]) if v.lower() == "active"}))
                    except (ValueError, IndexError):
                        continue

            self._t = threading.Thread(target=read, daemon=True)
            self._t.start()
        except Exception:
            self._proc = None
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._proc:
            time.sleep(0.1)
            self._proc.terminate()
            try:
                self._proc.wait(timeout=5)
            except Exception:
                self._proc.kill()
        if self._t:
            self._t.join(timeout=2)

    def summary(self) -> dict:
        sm = [x[0] for x in self.samples]
        mx = [x[1] for x in self.samples]
        reasons = set()
        for x in self.samples:
            reasons |= x[2]
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def ncu_traffic(kernel: str) -> float | None:
    """DRAM bytes per launch of `kernel` from the committed ncu summary, when present."""
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    try:
        return float(json.loads(p.read_text())[kernel]["dram_bytes_per_launch_full"])
    except Exception:
        return None


def cpu_baseline(workload: str, threads: int, sample_rows: int, reps: int = 3) -> dict:
    """The oracle (CPU restatement) on a bounded sample of the workload, all host threads."""
    import torch

    from oracle import pyoracle
    from polars_b200 import datagen

    maker = getattr(datagen, WORKLOADS[workload][0])
    t = maker(sample_rows, seed=99, device="cpu") if workload != "sort" else maker(sample_rows, seed=99, device="cpu")
    cols = datagen.to_numpy_columns(t)
    times = []
    pyoracle.groupby(cols, t.keys, t.aggs, t.predicate, n_threads=threads)  # warm-up
    for _ in range(reps):
        t0 = time.perf_counter()
        pyoracle.groupby(cols, t.keys, t.aggs, t.predicate, n_threads=threads)
        times.append(time.perf_counter() - t0)
    sec = statistics.median(times)
    del torch
    return {"value": sample_rows / sec, "unit": "rows/s", "cores": threads, "kind": "port",
            "sample": f"first {sample_rows:,} rows of the same generator (seed 99), median of {reps} after 1 warm-up"}


F64_RTOL, F64_ATOL = 1e-12, 1e-15  # float sums and means against the oracle's compensated sums


def _sorted_by_keys(res: dict, n_keys: int) -> list:
    """[(values, valid)] per column of a result dict, rows ordered by the keys (nulls first)."""
    import numpy as np

    from polars_b200 import _abi as A

    n = int(res["n_groups"])
    cols = []
    for dt, d, v in zip(res["dtypes"], res["data"], res["validity"]):
        vals = np.asarray(d)
        vals = np.unpackbits(vals.view(np.uint8), bitorder="little")[:n].astype(bool) if dt == A.BOOL else vals[:n]
        valid = np.unpackbits(np.asarray(v, dtype=np.uint8), bitorder="little")[:n].astype(bool)
        cols.append((vals, valid))
    sort_keys = []
    for j in reversed(range(n_keys)):
        vals, valid = cols[j]
        vv = np.where(valid, vals, np.zeros_like(vals))
        if vv.dtype.kind == "f":
            vv = vv.view(np.int32 if vv.dtype == np.float32 else np.int64)
        sort_keys += [vv, valid]
    order = np.lexsort(sort_keys) if n_keys and n else np.arange(n)
    return [(vals[order], valid[order]) for vals, valid in cols]


def compare_results(got: dict, want: dict, n_keys: int, aggs: list) -> dict:
    """The parity rules of the test suite, as figures: keys, counts, integer aggregates and min/max
    bit-exact; float64 sums and means within 1e-12 relative (+1e-15 absolute); float32 sums and
    means within 1 ulp of the oracle's float64 result rounded to float32."""
    import numpy as np

    out = {"checked": True, "groups": int(want["n_groups"]), "n_groups_equal": int(got["n_groups"]) == int(want["n_groups"]),
           "dtypes_equal": list(got["dtypes"]) == list(want["dtypes"]), "exact_int": True, "validity_equal": True,
           "max_rel_err_f64": 0.0, "max_ulps_f32": 0, "bad_values": 0}
    if not (out["n_groups_equal"] and out["dtypes_equal"]):
        out["ok"] = False
        return out
    g, w = _sorted_by_keys(got, n_keys), _sorted_by_keys(want, n_keys)
    ops = [None] * n_keys + [a[0] for a in aggs]
    for (gv, gval), (wv, wval), op in zip(g, w, ops):
        if not np.array_equal(gval, wval):
            out["validity_equal"] = False
            continue
        gv, wv = gv[wval], wv[wval]
        if gv.dtype.kind == "f" and op in ("Sum", "Mean"):
            nan = np.isnan(gv) & np.isnan(wv)
            if gv.dtype == np.float32:
                ia = gv.view(np.int32).astype(np.int64)
                ib = wv.astype(np.float32).view(np.int32).astype(np.int64)
                ia = np.where(ia < 0, -(ia & 0x7FFFFFFF), ia)
                ib = np.where(ib < 0, -(ib & 0x7FFFFFFF), ib)
                u = np.where(nan, 0, np.abs(ia - ib))
                out["max_ulps_f32"] = max(out["max_ulps_f32"], int(u.max()) if u.size else 0)
                out["bad_values"] += int((u > 1).sum())
            else:
                with np.errstate(invalid="ignore", divide="ignore"):
                    diff = np.where(nan | (gv == wv), 0.0, np.abs(gv - wv))
                    rel = np.where(diff == 0, 0.0, diff / np.maximum(np.abs(wv), F64_ATOL))
                out["max_rel_err_f64"] = max(out["max_rel_err_f64"], float(rel.max()) if rel.size else 0.0)
                out["bad_values"] += int((diff > F64_RTOL * np.abs(wv) + F64_ATOL).sum())
        else:
            same = (gv == wv) | (np.isnan(gv) & np.isnan(wv)) if gv.dtype.kind == "f" else (gv == wv)
            if not same.all():
                out["exact_int"] = False
                out["bad_values"] += int((~same).sum())
    out["ok"] = out["validity_equal"] and out["exact_int"] and out["bad_values"] == 0
    return out


def parity_against_oracle(got, table, threads: int) -> dict:
    """The CPU checker after the timed region: the oracle's group-by of the same table (copied to
    host memory) against the device result `got` (a host-output GroupByResult)."""
    from oracle import pyoracle
    from polars_b200 import datagen

    t0 = time.perf_counter()
    want = pyoracle.groupby(datagen.to_numpy_columns(table), table.keys, table.aggs, table.predicate,
                            n_threads=threads)
    g = {"n_groups": got.n_groups, "names": got.names, "dtypes": got.dtypes, "data": got.data,
         "validity": got.validity}
    rep = compare_results(g, want, len(table.keys), table.aggs)
    rep["rows"] = table.n_rows
    rep["oracle_s"] = time.perf_counter() - t0
    return rep


def filter_subrecord(t, cols, h, stream, threads: int | None) -> dict:
    """The top-level filter of the hash workload (every column compacted by the predicate, one
    pass) and the u8 -> u32 inclusive scan over 100M keep bytes, on device-resident inputs: device
    time, the dominant kernel's HBM roofline, and (with `threads`) parity against the oracle."""
    import numpy as np
    import torch

    from polars_b200._native import filter_columns

    n = t.n_rows

    def call():
        return filter_columns(cols, t.predicate, output="device", handle=h)
    res = call()
    ms = time_calls(call, stream, 5, 2)
    h.set_profiling(True)
    call()
    st = h.last_stats()
    h.set_profiling(False)
    kern = {k: rec["ms"] for k, rec in st["kernels"].items()}
    kept = int(res.n_groups)
    in_bytes = t.bytes_per_row() * n
    out_bytes = kept * sum(d.element_size() + (1.0 / 8.0 if v is not None else 0.0) for d, v in t.columns.values())
    peak, peak_kind = load_peaks()
    dom = max(kern, key=kern.get)
    rec = {"workload": "top-level filter (v1>-0.5)&(v3%7!=0) of the hash workload's 100M rows, 4 columns compacted",
           "rows": n, "kept": kept, "ms_per_step": ms, "rows_per_s": n / (ms / 1e3), "kernels_ms": kern,
           "roofline": {"kernel": dom, "algorithmic_bytes": in_bytes + out_bytes,
                        "achieved": (in_bytes + out_bytes) / (kern[dom] / 1e3) / 1e9, "peak": peak,
                        "frac": (in_bytes + out_bytes) / (kern[dom] / 1e3) / 1e9 / peak, "peak_kind": peak_kind},
           "parity": None}
    # the u8 -> u32 inclusive scan (the reference's MLX cumsum), 100M device bytes in, 400 MB out
    dev = next(iter(t.columns.values()))[0].device
    g = torch.Generator(device=dev)
    g.manual_seed(5)
    u8 = torch.randint(0, 256, (n,), dtype=torch.uint8, device=dev, generator=g)
    o32 = torch.empty(n, dtype=torch.int32, device=u8.device)

    def scan():
        h.check(h._lib.pmb_cumsum_u8_to_u32(h.raw, u8.data_ptr(), o32.data_ptr(), n, 1))
    ms_scan = time_calls(scan, stream, 5, 2)
    h.set_profiling(True)
    scan()
    kscan = {k: r["ms"] for k, r in h.last_stats()["kernels"].items()}
    h.set_profiling(False)
    sdom = max(kscan, key=kscan.get)
    rec["scan"] = {"rows": n, "ms_per_step": ms_scan, "kernels_ms": kscan,
                   "roofline": {"kernel": sdom, "algorithmic_bytes": 5 * n,
                                "achieved": 5 * n / (kscan[sdom] / 1e3) / 1e9, "peak": peak,
                                "frac": 5 * n / (kscan[sdom] / 1e3) / 1e9 / peak}}
    if threads:
        from oracle import pyoracle
        from polars_b200 import datagen

        t0 = time.perf_counter()
        host_cols = datagen.to_numpy_columns(t)
        keep = pyoracle.filter_mask(host_cols, t.predicate, n_threads=threads)
        got = filter_columns(cols, t.predicate, output="host", handle=h)
        ok = int(got.n_groups) == int(keep.sum())
        bad_cols = []
        for j, name in enumerate(got.names):
            d, v = host_cols[name]
            want = d[keep]
            gd = np.asarray(got.data[j])[: got.n_groups]
            gv = np.unpackbits(np.asarray(got.validity[j], dtype=np.uint8), bitorder="little")[: got.n_groups].astype(bool)
            wv = np.ones(want.size, bool) if v is None else np.unpackbits(v, bitorder="little")[:n].astype(bool)[keep]
            if not (np.array_equal(gv, wv) and np.array_equal(gd[wv].view(np.uint8), want[wv].view(np.uint8))):
                bad_cols.append(name)
        scan_ok = bool(np.array_equal(o32.cpu().numpy().view(np.uint32), pyoracle.cumsum_u8_to_u32(u8.cpu().numpy())))
        rec["parity"] = {"checked": True, "rows": n, "kept_equal": ok, "bit_exact_columns": not bad_cols,
                         "bad_columns": bad_cols, "scan_bit_exact": scan_ok, "ok": ok and not bad_cols and scan_ok,
                         "oracle_s": time.perf_counter() - t0}
    del u8, o32
    return rec


def sort_extras(t, cols, h, stream, strategy: str, used: str, ms_group_by: float):
    """The sort workload's LSD radix sort + segmented reduce strategy (when AUTO picked another)
    and the group-by with its result sorted by the keys on the device in the same call (a Sort
    over a GroupBy), with the kernels of one profiled call."""
    from polars_b200._native import groupby

    n = t.n_rows
    sort_strategy = None
    if used != "sort":
        ms_sort = time_calls(lambda: groupby(cols, t.keys, t.aggs, t.predicate, strategy="sort", output="device",
                                             handle=h), stream, 3, 1)
        sort_strategy = {"strategy": "sort", "ms_per_step": ms_sort, "rows_per_s": n / (ms_sort / 1e3)}

    def sorted_call():
        return groupby(cols, t.keys, t.aggs, t.predicate, strategy=strategy, output="device", handle=h,
                       sort={"by": list(t.keys)})
    ms_sorted = time_calls(sorted_call, stream, 3, 1)
    h.set_profiling(True)
    sorted_call()
    st = h.last_stats()
    h.set_profiling(False)
    sorted_output = {"by": list(t.keys), "ms_per_step": ms_sorted, "ms_group_by_alone": ms_group_by,
                     "rows_per_s": n / (ms_sorted / 1e3), "kernels_ms": {k: rec["ms"] for k, rec in st["kernels"].items()}}
    return sort_strategy, sorted_output


def sort_parity_slice(got, table, threads: int, k2: int = 0) -> dict:
    """Parity of the sort workload's group-by over one slice of its key space: the groups whose
    second key equals `k2` are exactly the groups of the rows with that key, so the oracle's group-by
    of those rows (1/64 of all rows) must equal the device result's groups with k2 == `k2`. Exact,
    and a few seconds of CPU instead of the minutes of a 49M-group oracle run."""
    import numpy as np

    from oracle import pyoracle

    t0 = time.perf_counter()
    mask = table.columns["k2"][0] == k2
    cols = {name: (d[mask].cpu().numpy(), None) for name, (d, v) in table.columns.items()}
    want = pyoracle.groupby(cols, table.keys, table.aggs, None, n_threads=threads)
    kcol = got.names.index("k2")
    n = int(got.n_groups)
    sel = np.nonzero(np.asarray(got.data[kcol])[:n] == k2)[0]
    data, valid = [], []
    for d, v in zip(got.data, got.validity):
        data.append(np.asarray(d)[:n][sel])
        bits = np.unpackbits(np.asarray(v, dtype=np.uint8), bitorder="little")[:n][sel]
        valid.append(np.packbits(bits, bitorder="little"))
    g = {"n_groups": len(sel), "names": got.names, "dtypes": got.dtypes, "data": data, "validity": valid}
    rep = compare_results(g, want, len(table.keys), table.aggs)
    rep["rows"] = int(mask.sum().item())
    rep["slice"] = f"k2 == {k2}: 1/64 of the rows and of the groups"
    rep["oracle_s"] = time.perf_counter() - t0
    return rep


def sort_subrecord(device, h, stream, threads: int | None) -> dict:
    """The sort workload (200M rows, two-column key, ~49M groups) on device-resident inputs: AUTO
    (the partitioned strategy), the sort strategy, the sorted group-by, its dominant kernel against
    the HBM roofline, and (with `threads`) parity of the AUTO result against the oracle."""
    import torch

    from polars_b200 import datagen
    from polars_b200._native import groupby

    n = WORKLOADS["sort"][1]
    t = datagen.make_sort(n, seed=1234, device=device)
    torch.cuda.synchronize()
    cols = datagen.to_column_data(t)

    def call():
        return groupby(cols, t.keys, t.aggs, None, output="device", handle=h)
    r = call()
    ms = time_calls(call, stream, 5, 2)
    h.set_profiling(True)
    call()
    st = h.last_stats()
    h.set_profiling(False)
    kern = {k: rec["ms"] for k, rec in st["kernels"].items()}
    peak, peak_kind = load_peaks()
    bpr = t.bytes_per_row()
    sort_strategy, sorted_output = sort_extras(t, cols, h, stream, "auto", r.strategy, ms)
    rec = {"workload": WORKLOADS["sort"][2], "rows": n, "groups": r.n_groups, "strategy": r.strategy,
           "ms_per_step": ms, "rows_per_s": n / (ms / 1e3), "bytes_per_row": bpr,
           "pipeline_frac": (bpr * n / (ms / 1e3) / 1e9) / peak, "peak_kind": peak_kind, "kernels_ms": kern,
           "sort_strategy": sort_strategy, "sorted_output": sorted_output, "parity": None}
    if threads:
        got = groupby(cols, t.keys, t.aggs, None, output="host", handle=h)
        rec["parity"] = sort_parity_slice(got, t, threads)
        del got
    del cols, t
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return rec


def batch_queries(device, seed: int, stop_rows: int | None = None, max_total: int = BATCH_ROWS):
    """The batched workload's tables and their (columns, keys, aggs, predicate) tuples."""
    from polars_b200 import datagen

    tables = datagen.make_batch(BATCH_QUERIES, seed=seed, device=device, max_total=max_total, stop_rows=stop_rows)
    return tables, [(datagen.to_column_data(t), t.keys, t.aggs, t.predicate) for t in tables]


def time_calls(fn, stream, steps: int, warmup: int) -> float:
    """ms per call of fn(), CUDA events on `stream`. The library calls synchronise before they
    return, so the events bracket their host work too."""
    import torch

    for _ in range(warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def batch_vs_plain(qs, rows: int, stream, h_learned, h_plain, steps: int = 3, plain_steps: int = 2) -> dict:
    """Batched + learned selector against three other forms of the same queries: batched with the
    plain cardinality heuristic (the selector's share), the plain loop in C (one pmb_groupby per
    query inside the library, host outputs: the batching's share) and the plain loop in Python
    (one ctypes groupby call per query, device outputs: adds the binding's per-call cost)."""
    from polars_b200._native import groupby, groupby_batched, prepare_batched

    # the batched calls pass a batch prepared once (its C arguments marshalled before timing)
    prep_dev = prepare_batched(qs, output="device")
    prep_host = prepare_batched(qs, output="host")

    def plain():
        for c, k, a, p in qs:
            groupby(c, k, a, p, output="device", handle=h_plain)

    def c_loop():
        h_plain.set_batching(False)
        try:
            groupby_batched(prep_host, handle=h_plain)
        finally:
            h_plain.set_batching(True)

    ms_b = time_calls(lambda: groupby_batched(prep_dev, handle=h_learned), stream, steps, 3)
    ms_bh = time_calls(lambda: groupby_batched(prep_dev, handle=h_plain), stream, steps, 3)
    ms_bhh = time_calls(lambda: groupby_batched(prep_host, handle=h_plain), stream, plain_steps, 1)
    ms_c = time_calls(c_loop, stream, plain_steps, 1)
    ms_p = time_calls(plain, stream, plain_steps, 1)
    arm = lambda ms, st: {"rows_per_s": rows / (ms / 1e3), "ms_per_step": ms, "steps": st}  # noqa: E731
    return {"workload": BATCH_DESC, "queries": len(qs), "rows": rows,
            "batched_learned": arm(ms_b, steps), "batched_heuristic": arm(ms_bh, steps),
            "batched_heuristic_host": arm(ms_bhh, plain_steps), "plain_loop_c": arm(ms_c, plain_steps),
            "plain_heuristic": arm(ms_p, plain_steps),
            "speedup": ms_p / ms_b, "speedup_vs_c_loop": ms_c / ms_bhh, "selector_gain": ms_bh / ms_b,
            "note": "the batched arms and the C loop take a batch prepared once before timing (prepare_batched: "
                    "its C arguments built once); the Python loop makes one groupby call per query with device "
                    "outputs; the C loop has host outputs only, so speedup_vs_c_loop divides it by the batched "
                    "heuristic arm with host outputs (batched_heuristic_host): the batching's own share"}


def batch_parity(tables, qs, h, threads: int) -> dict:
    """The checker after the timed region: every query of the batch through pmb_groupby_batched
    (host outputs) against the oracle's group-by of the same query."""
    from oracle import pyoracle
    from polars_b200 import datagen
    from polars_b200._native import groupby_batched

    t0 = time.perf_counter()
    res = groupby_batched(qs, output="host", handle=h)
    agg = {"checked": True, "queries": len(tables), "rows": sum(t.n_rows for t in tables), "ok": True,
           "exact_int": True, "validity_equal": True, "max_rel_err_f64": 0.0, "bad_values": 0, "failed_queries": 0}
    for t, got in zip(tables, res):
        want = pyoracle.groupby(datagen.to_numpy_columns(t), t.keys, t.aggs, t.predicate, n_threads=threads)
        g = {"n_groups": got.n_groups, "names": got.names, "dtypes": got.dtypes, "data": got.data,
             "validity": got.validity}
        rep = compare_results(g, want, len(t.keys), t.aggs)
        if not rep["ok"]:
            agg["failed_queries"] += 1
            agg["ok"] = False
        for k in ("exact_int", "validity_equal"):
            agg[k] = agg[k] and rep.get(k, False)
        agg["max_rel_err_f64"] = max(agg["max_rel_err_f64"], rep.get("max_rel_err_f64", 0.0))
        agg["bad_values"] += rep.get("bad_values", 0)
    agg["oracle_s"] = time.perf_counter() - t0
    return agg


def batch_cpu_sample(threads: int, stop_rows: int, reps: int = 3) -> tuple[float, int, int]:
    """The oracle over the batched workload's leading queries (CPU-generated, same generator):
    (seconds per pass, rows, queries), median of `reps` after one warm-up."""
    from oracle import pyoracle
    from polars_b200 import datagen

    tables = datagen.make_batch(BATCH_QUERIES, seed=4, device="cpu", max_total=BATCH_ROWS, stop_rows=stop_rows)
    cols = [datagen.to_numpy_columns(t) for t in tables]

    def one():
        for t, c in zip(tables, cols):
            pyoracle.groupby(c, t.keys, t.aggs, t.predicate, n_threads=threads)

    one()
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        one()
        times.append(time.perf_counter() - t0)
    return statistics.median(times), sum(t.n_rows for t in tables), len(tables)


def run_reference(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = len(os.sched_getaffinity(0))
    from oracle import pyoracle
    from polars_b200 import datagen

    if args.workload == "batch":
        sec, rows, nq = batch_cpu_sample(threads, 10_000_000, reps=max(1, args.steps))
        value = rows / sec
        line = {
            "impl": "reference", "metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": BATCH_DESC, "rows_per_step": rows,
                       "note": "CPU restatement of the reference algorithm (oracle/oracle.cpp), one call per query; "
                               "the reference is Rust+Metal and cannot run here"},
            "cpu_baseline": {"value": value, "unit": "rows/s", "cores": threads, "kind": "port",
                             "sample": f"the leading {nq} queries ({rows:,} rows) of the batch, CPU-generated, median"},
            "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line), flush=True)
        return
    sample = {"hash": 20_000_000, "small": 1_000_000, "sort": 20_000_000}[args.workload]
    maker = getattr(datagen, WORKLOADS[args.workload][0])
    t = maker(sample, seed=99, device="cpu")
    cols = datagen.to_numpy_columns(t)
    for _ in range(args.warmup):
        pyoracle.groupby(cols, t.keys, t.aggs, t.predicate, n_threads=threads)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        pyoracle.groupby(cols, t.keys, t.aggs, t.predicate, n_threads=threads)
        times.append(time.perf_counter() - t0)
    ms = 1e3 * sum(times) / len(times)
    value = sample / (ms / 1e3)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOADS[args.workload][2], "rows_per_step": sample,
                   "note": "CPU restatement of the reference algorithm (oracle/oracle.cpp); the reference is Rust+Metal "
                           "and cannot run here. Each step is a bounded sample (the first rows of the same "
                           "generator) rather than all rows of the workload, so that --steps K --warmup W ends "
                           "within minutes (the oracle needs ~8 s per 100M rows on 16 threads); rows/s is "
                           "per row, and the ours-arm line's parity check times the oracle on all rows "
                           "(parity.oracle_s)"},
        "cpu_baseline": {"value": value, "unit": "rows/s", "cores": threads, "kind": "port",
                         "sample": f"first {sample:,} rows of the workload generator (seed 99) per step"},
        "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="hash", choices=sorted(WORKLOADS) + ["batch"])
    ap.add_argument("--no-batched", action="store_true", help="leave out the batched-vs-plain comparison")
    ap.add_argument("--strategy", default="auto", help="group-by strategy of the timed calls (default: auto)")
    ap.add_argument("--rows", type=int, default=0,
                    help="override the workload's row count (batch: the total over its 4096 queries)")
    ap.add_argument("--e2e-steps", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true", help="leave out the CPU legs: baseline and parity check")
    ap.add_argument("--no-sort", action="store_true", help="leave the sort workload out of the default line")
    ap.add_argument("--no-filter", action="store_true", help="leave the top-level filter out of the default line")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        run_reference(args)
        return

    import torch

    from polars_b200 import datagen
    from polars_b200._native import ColumnData, Handle, groupby
    from polars_b200.replicas import barrier, dist_env, reduce_step_stats

    rank, local_rank, world = dist_env()
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta

        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local_rank))
    device = torch.device("cuda", local_rank)
    torch.cuda.set_device(device)
    if args.workload == "batch":
        run_batch(args, device, rank, local_rank, world)
        return

    maker_name, default_rows, desc = WORKLOADS[args.workload]
    n = args.rows or default_rows
    t = getattr(datagen, maker_name)(n, seed=1234 + rank, device=device)
    torch.cuda.synchronize()
    cols = datagen.to_column_data(t)
    bytes_per_row = t.bytes_per_row()

    h = Handle(local_rank)
    stream = torch.cuda.current_stream(device)
    h.set_stream(stream.cuda_stream)

    def step(profile: bool):
        return groupby(cols, t.keys, t.aggs, t.predicate, strategy=args.strategy, output="device", handle=h)

    for _ in range(args.warmup):
        r = step(False)
    n_groups = r.n_groups

    # timed region: device-resident inputs, profiling events around every kernel
    h.set_profiling(True)
    barrier(device)
    torch.cuda.synchronize()
    kern_ms: dict[str, list] = {}
    launches = 0
    with ClockSampler(local_rank) as clk:
        ev0 = torch.cuda.Event(enable_timing=True)
        ev1 = torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for _ in range(args.steps):
            step(True)
            st = h.last_stats()
            launches += st["kernel_launches"]
            for name, rec in st["kernels"].items():
                kern_ms.setdefault(name, []).append((rec["ms"], rec["launches"]))
        ev1.record(stream)
        torch.cuda.synchronize()
    barrier(device)
    total_ms = ev0.elapsed_time(ev1)
    ms_step = total_ms / args.steps
    ms_max, rows_all = reduce_step_stats(ms_step, n, device)
    value = rows_all / (ms_max / 1e3)

    # dominant kernel roofline
    peak, peak_kind = load_peaks()
    dom = max(kern_ms, key=lambda k: sum(x[0] for x in kern_ms[k]))
    dom_ms = sum(x[0] for x in kern_ms[dom]) / sum(x[1] for x in kern_ms[dom])
    alg_bytes = bytes_per_row * n
    achieved = alg_bytes / (dom_ms / 1e3) / 1e9
    h.set_profiling(False)

    # end to end through the public API: pinned host inputs, host outputs
    e2e = None
    if rank == 0 or world > 1:
        host = {}
        for name, c in cols.items():
            hd = torch.empty(c.data.shape, dtype=c.data.dtype, pin_memory=True)
            hd.copy_(c.data)
            hv = None
            if c.validity is not None:
                hv = torch.empty(c.validity.shape, dtype=c.validity.dtype, pin_memory=True)
                hv.copy_(c.validity)
            host[name] = ColumnData(hd, hv, dtype=c.dtype, length=c.length)
        e2e_steps = args.e2e_steps or max(3, min(args.steps, 5))
        for _ in range(max(3, args.warmup)):
            groupby(host, t.keys, t.aggs, t.predicate, strategy=args.strategy, output="host", handle=h)
        h.set_profiling(True)
        groupby(host, t.keys, t.aggs, t.predicate, strategy=args.strategy, output="host", handle=h)
        io = h.last_stats()
        h.set_profiling(False)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(e2e_steps):
            groupby(host, t.keys, t.aggs, t.predicate, strategy=args.strategy, output="host", handle=h)
        torch.cuda.synchronize()
        e2e_ms = 1e3 * (time.perf_counter() - t0) / e2e_steps
        e2e_ms_max, rows_e2e = reduce_step_stats(e2e_ms, n, device)
        e2e = {"value": rows_e2e / (e2e_ms_max / 1e3), "unit": "rows/s", "h2d_bytes_per_step": int(io["h2d_bytes"]),
               "d2h_bytes_per_step": int(io["d2h_bytes"]), "ms_per_step": e2e_ms_max, "steps": e2e_steps}

    cpu = None
    parity = None
    if rank == 0 and not args.no_cpu_baseline:
        threads = len(os.sched_getaffinity(0))
        sample = {"hash": 10_000_000, "small": 1_000_000, "sort": 10_000_000}[args.workload]
        cpu = cpu_baseline(args.workload, threads, sample)
        # the checker, after the timed region: the same call's result against the oracle over all rows
        got = groupby(cols, t.keys, t.aggs, t.predicate, strategy=args.strategy, output="host", handle=h)
        parity = parity_against_oracle(got, t, threads)
        del got

    filt = None
    if args.workload == "hash" and not args.no_filter:
        filt = filter_subrecord(t, cols, h, stream, None if args.no_cpu_baseline else len(os.sched_getaffinity(0)))

    sort_strategy = sorted_output = None
    if args.workload == "sort":
        sort_strategy, sorted_output = sort_extras(t, cols, h, stream, args.strategy, r.strategy, ms_max)

    # the default line also carries the sort workload (200M rows, ~49M groups) as a sub-record
    sort_rec = None
    if args.workload == "hash" and not args.no_sort and world == 1:
        del cols, t
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
        sort_rec = sort_subrecord(device, h, stream, None if args.no_cpu_baseline else len(os.sched_getaffinity(0)))

    batched = None
    if not args.no_batched and args.workload == "hash":
        tables_b, qs_b = batch_queries(device, seed=4 + rank)
        torch.cuda.synchronize()
        h_plain = Handle(local_rank, selector=None)
        h_plain.set_stream(stream.cuda_stream)
        batched = batch_vs_plain(qs_b, sum(tb.n_rows for tb in tables_b), stream, h, h_plain)
        h_plain.close()
        if not args.no_cpu_baseline:
            batched["parity"] = batch_parity(tables_b, qs_b, h, len(os.sched_getaffinity(0)))
        del tables_b, qs_b

    if rank == 0:
        clocks = clk.summary()
        line = {
            "metric": METRIC,
            "value": value,
            "unit": "rows/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms_max,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic",
            "config": {"workload": desc, "rows_per_gpu": n, "groups": n_groups, "strategy": r.strategy,
                       "capacity": r.capacity, "rehash_count": r.rehash_count,
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": (f"inputs {alg_bytes / 1e9:.2f} GB per GPU > 126 MB L2, no flush needed"
                              if alg_bytes > 126e6 else
                              f"inputs {alg_bytes / 1e6:.1f} MB per GPU fit in the 126 MB L2: timed warm, no flush "
                              "(the 100M- and 200M-row workloads exceed L2)"),
                       "bytes_per_row": bytes_per_row},
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": ncu_traffic(dom) if args.workload == "hash" and n == default_rows else None,
                         "algorithmic_bytes_per_launch": alg_bytes, "avg_launch_ms": dom_ms,
                         "pipeline_frac": (alg_bytes / (ms_step / 1e3) / 1e9) / peak},
            "kernels_ms_per_step": {k: sum(x[0] for x in v) / args.steps for k, v in kern_ms.items()},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clocks,
            "parity": parity,
            "filter": filt,
            "batched": batched,
            "sort_strategy": sort_strategy,
            "sorted_output": sorted_output,
            "sort": sort_rec,
        }
        print(json.dumps(line), flush=True)
    h.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


def run_batch(args, device, rank: int, local_rank: int, world: int) -> None:
    """--workload batch: the headline is pmb_groupby_batched with the learned selector."""
    import torch

    from polars_b200._native import ColumnData, Handle, groupby_batched, prepare_batched
    from polars_b200.replicas import barrier, reduce_step_stats

    tables, qs = batch_queries(device, seed=4 + rank, max_total=args.rows or BATCH_ROWS)
    torch.cuda.synchronize()
    rows = sum(t.n_rows for t in tables)
    bytes_per_row = tables[0].bytes_per_row()
    alg_bytes = bytes_per_row * rows
    stream = torch.cuda.current_stream(device)
    h = Handle(local_rank)
    h.set_stream(stream.cuda_stream)

    prep = prepare_batched(qs, output="device")  # C arguments marshalled once, before timing

    def step():
        return groupby_batched(prep, handle=h)

    for _ in range(args.warmup):
        res = step()
    barrier(device)
    torch.cuda.synchronize()
    with ClockSampler(local_rank) as clk:
        ms = time_calls(step, stream, args.steps, 0)
    launches = h.last_stats()["kernel_launches"] * args.steps
    barrier(device)
    ms_max, rows_all = reduce_step_stats(ms, rows, device)
    value = rows_all / (ms_max / 1e3)
    # one profiled call (the same launches run eagerly, an event pair around each kernel)
    h.set_profiling(True)
    step()
    st = h.last_stats()
    h.set_profiling(False)
    kern = {k: v["ms"] for k, v in st["kernels"].items()}
    # every launch of the batched kernel in one call (a first round, and a second one for the queries
    # whose tables overflowed) together reads the batch's bytes once: divide by their summed time
    agg_ms = st["kernels"]["batch_agg"]["ms"]
    agg_launches = st["kernels"]["batch_agg"]["launches"]
    peak, peak_kind = load_peaks()
    achieved = alg_bytes / (agg_ms / 1e3) / 1e9
    groups = sum(r.n_groups for r in res)

    # end to end: every query's columns in pinned host memory, results copied back
    host_qs = []
    for c, k, a, p in qs:
        hc = {}
        for name, col in c.items():
            hd = torch.empty(col.data.shape, dtype=col.data.dtype, pin_memory=True)
            hd.copy_(col.data)
            hv = None
            if col.validity is not None:
                hv = torch.empty(col.validity.shape, dtype=col.validity.dtype, pin_memory=True)
                hv.copy_(col.validity)
            hc[name] = ColumnData(hd, hv, dtype=col.dtype, length=col.length)
        host_qs.append((hc, k, a, p))
    groupby_batched(host_qs, output="host", handle=h)
    h.set_profiling(True)
    groupby_batched(host_qs, output="host", handle=h)
    io = h.last_stats()
    h.set_profiling(False)
    e2e_steps = args.e2e_steps or 3
    e2e_ms = time_calls(lambda: groupby_batched(host_qs, output="host", handle=h), stream, e2e_steps, 0)
    e2e_ms_max, rows_e2e = reduce_step_stats(e2e_ms, rows, device)
    del host_qs

    h_plain = Handle(local_rank, selector=None)
    h_plain.set_stream(stream.cuda_stream)
    cmp = batch_vs_plain(qs, rows, stream, h, h_plain, steps=args.steps)
    h_plain.close()
    parity = None
    if rank == 0 and not args.no_cpu_baseline:
        parity = batch_parity(tables, qs, h, len(os.sched_getaffinity(0)))

    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        threads = len(os.sched_getaffinity(0))
        sec, srows, snq = batch_cpu_sample(threads, 10_000_000)
        cpu = {"value": srows / sec, "unit": "rows/s", "cores": threads, "kind": "port",
               "sample": f"the leading {snq} queries ({srows:,} rows) of the batch, CPU-generated, oracle one call per "
                         f"query, median of 3 after 1 warm-up"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": BATCH_DESC, "queries": len(qs), "rows_per_gpu": rows, "groups": groups,
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "l2": f"inputs {alg_bytes / 1e9:.2f} GB per GPU > 126 MB L2, no flush needed",
                       "bytes_per_row": bytes_per_row, "selector": "learned (shipped parameters)"},
            "roofline": {"bound": "hbm", "kernel": "batch_agg", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind, "traffic": ncu_traffic("batch_agg"),
                         "algorithmic_bytes_per_call": alg_bytes, "launches_per_call": agg_launches,
                         "summed_launch_ms": agg_ms,
                         "pipeline_frac": (alg_bytes / (ms / 1e3) / 1e9) / peak},
            "kernels_ms_per_step": kern,
            "cpu_baseline": cpu,
            "e2e": {"value": rows_e2e / (e2e_ms_max / 1e3), "unit": "rows/s", "h2d_bytes_per_step": int(io["h2d_bytes"]),
                    "d2h_bytes_per_step": int(io["d2h_bytes"]), "ms_per_step": e2e_ms_max, "steps": e2e_steps},
            "gpu_launches": launches,
            "clocks": clk.summary(),
            "vs_plain": cmp,
            "parity": parity,
        }
        print(json.dumps(line), flush=True)
    h.close()
    if world > 1:
        import torch.distributed as dist

        dist.destroy_process_group()


if __name__ == "__main__":
    main()
