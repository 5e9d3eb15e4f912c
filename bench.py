"""Benchmark of the B200 join + runtime-filter + aggregate path.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload star|join|agg|serve|grace|parquet] [--scale S]

Default workload (`star`): the star join with runtime Bloom filters --
fact 300M rows {fk_a in [0, 20M), fk_b in [0, 1M), price, discount}, dim_a
20M and dim_b 1M rows with a 5%-selective int32 predicate and a 25-value int32
attribute; a blocked Bloom filter per filtered dimension applied to the fact
scan, a two-join probe and GROUP BY dim_a.attr SUM(price * (1 - discount)).
One step = one whole query (both dimension builds with their filters, the
fact probe, the grouped result). The metric is fact rows per second
(Mrows/s, higher is better).

With --gpus N > 1 (torchrun, one process per GPU) every rank runs the query
on its own shard of the fact stream (different fact rows, the same
dimensions): weak scaling, no collective on the data path; the step time is
the max over ranks.

Inputs are generated on the device by the library's counter-based generators
(synthetic, seeded). `value` is measured with inputs resident in HBM; `e2e`
runs the same query through the C ABI with host Arrow buffers (pinned), the
host-to-device copies inside the timed region. The fact columns (9.6 GB)
exceed the 126 MB L2, so no L2 flush is needed between steps.

--impl reference times the reference algorithm restated in C (the CPU oracle,
multi-threaded over all host cores) on a bounded sample of the same workload.
"""
from __future__ import annotations

import argparse
import importlib
import json
import os
import shutil
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def hbm_peak():
    try:
        with open(PEAKS) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# ---- clocks during the timed region ------------------------------------------------------
class Clocks:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.samples = []
        self.proc = None

    def __enter__(self):
        exe = shutil.which("nvidia-smi")
        if exe:
            self.proc = subprocess.Popen([exe, "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.reader = threading.Thread(target=self._read, daemon=True)
            self.reader.start()
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 7:
                self.samples.append(parts)

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.15)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if s[3 + i].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ---- distributed plumbing ----------------------------------------------------------------
def dist_init(n_gpus):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    return rank, world, local, pg


def star_config(scale, fact_scale):
    """The star workload's description, the same for both arms."""
    nf = int(300_000_000 * fact_scale)
    return {"workload": "star join + runtime Bloom filters + GROUP BY attr SUM(price*(1-discount))",
            "fact_rows_per_gpu": nf, "dim_a_rows": int(20_000_000 * scale), "dim_b_rows": int(1_000_000 * scale),
            "selectivity": "5% per dimension", "groups": 25,
            "l2": f"inputs ({nf * 32 / 1e9:.1f} GB per GPU) larger than L2; no flush"}


def barrier(pg):
    if pg is not None:
        pg.barrier()


def max_over_ranks(pg, value, device):
    return _shard().max_over_ranks(pg, value, device)


def _shard():
    return importlib.import_module("krishiv-engine_b200.shard")


# ---- the CPU baseline (the oracle's multi-threaded restatement) ---------------------------
def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    return O


def host_bytes_available():
    try:
        import psutil
        return int(psutil.virtual_memory().available)
    except Exception:
        return 0


def cpu_star_inputs(scale, fact_scale, threads):
    """The star query's whole input on the host, generated by the oracle's
    counter-based generators (the device generators' functions) on `threads`
    host threads; None when the host has too little free memory for it."""
    O = _oracle()
    W = importlib.import_module("krishiv-engine_b200.workloads")
    nf = int(300_000_000 * fact_scale)
    need = 32 * nf + 16 * int(20_000_000 * scale)
    if host_bytes_available() < 2 * need:
        return None
    fact, dims = O.star_inputs_mt(scale, W.STAR_SEED, threads, fact_rows=nf, pred=W.PRED_VALUE)
    return fact, dims


def cpu_star_full(fact, dims, threads, runs):
    """The CPU oracle's star query (dimension builds with their key filters,
    the fact probe split over `threads` host threads, compensated group sums)
    over every fact row given, `runs` times: (median whole-query seconds,
    the last answer)."""
    O = _oracle()
    W = importlib.import_module("krishiv-engine_b200.workloads")
    times, ans = [], None
    for _ in range(runs):
        t0 = time.perf_counter()
        ans = O.star_query(fact, dims, pred=W.PRED_VALUE, threads=threads)
        times.append(time.perf_counter() - t0)
    return statistics.median(times), ans


def cpu_star(scale, sample_rows, threads, seed=None):
    """Times the star query on the host cores with the CPU oracle on the first
    `sample_rows` fact rows (dimensions at full size); returns the whole-query
    rate extrapolated to the full fact table (build time + full probe). Used
    only when the host cannot hold the whole fact table."""
    O = _oracle()
    W = importlib.import_module("krishiv-engine_b200.workloads")
    seed = W.STAR_SEED if seed is None else seed
    nf = int(300_000_000 * scale)
    s = min(sample_rows, nf)
    fact, dims = O.star_inputs_mt(scale, seed, threads, fact_rows=s, pred=W.PRED_VALUE)
    groups, passed, joined, tb, tp = O.star_query(fact, dims, pred=W.PRED_VALUE, threads=threads)
    probe_rate = s / tp
    whole = tb + nf / probe_rate
    return {"value": nf / whole / 1e6, "build_s": tb, "probe_rows_per_s": probe_rate, "sample_rows": s,
            "threads": threads, "groups": len(groups), "joined": joined}


def star_parity(gpu_groups, gpu_counters, oracle_answer, rows, tol=1e-12):
    """The GPU's answer against the oracle's on the same rows: the rows passing
    both key filters and the joined rows exactly, the same groups, and each
    group's sum within `tol` relative of the oracle's compensated sum."""
    groups, passed, joined, _, _ = oracle_answer
    worst = 0.0
    for k, (want, _) in groups.items():
        got = gpu_groups.get(k)
        if got is None:
            worst = float("inf")
            break
        worst = max(worst, abs(got - want) / max(abs(want), 1e-300))
    same_groups = sorted(groups) == sorted(gpu_groups)
    ok = (passed == gpu_counters["passed_filters"] and joined == gpu_counters["joined_rows"] and same_groups
          and worst <= tol)
    return {"checker": "CPU oracle star query (the reference's algorithms restated in C) on the same rows",
            "fact_rows": rows, "passed_filters": [gpu_counters["passed_filters"], passed],
            "joined_rows": [gpu_counters["joined_rows"], joined], "groups": [len(gpu_groups), len(groups)],
            "max_rel_err": worst, "tolerance": tol, "ok": bool(ok)}


def cpu_join(scale, threads=1):
    """The oracle's hash join (single thread) on the whole plain-join workload:
    build + probe rows per second."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    W = importlib.import_module("krishiv-engine_b200.workloads")
    nb, np_ = int(1_000_000 * scale), int(10_000_000 * scale)
    bk, _ = O.gen_column(3, W.JOIN_SEED, 1, nb, lo=0, hi=nb)
    pk, _ = O.gen_column(0, W.JOIN_SEED, 3, np_, lo=0, hi=2 * nb - 1)
    t0 = time.perf_counter()
    p, b = O.hash_join(0, [(bk, None)], [(pk, None)])
    dt = time.perf_counter() - t0
    return {"value": (nb + np_) / dt / 1e6, "rows_out": int(p.size), "seconds": dt}


def cpu_agg(scale, sample):
    """The oracle's grouped aggregate (single thread) over the first `sample`
    rows of the aggregate workload, 15 aggregates: rows per second."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    W = importlib.import_module("krishiv-engine_b200.workloads")
    n = min(sample, int(100_000_000 * scale))
    seed = W.AGG_SEED
    k, _ = O.gen_column(4, seed, 1, n, lo=0, hi=1_000_000, x0=1.1)
    dec, dv = O.gen_column(0, seed, 2, n, lo=100, hi=10_000_000, null_fraction=0.02)
    f, fv = O.gen_column(2, seed, 3, n, x0=0.0, x1=1.0, null_fraction=0.02)
    q, qv = O.gen_column(1, seed, 4, n, lo=1, hi=50, null_fraction=0.02)
    cols = [{"values": dec, "valid": dv, "type": O.T_DEC64, "precision": 15, "scale": 2},
            {"values": f, "valid": fv, "type": O.T_F64}, {"values": q, "valid": qv, "type": O.T_I32}]
    exprs = [(fn, c) for c in range(3) for fn in (O.SUM, O.COUNT, O.MIN, O.MAX, O.AVG)]
    t0 = time.perf_counter()
    O.hash_aggregate(k, None, cols, exprs)
    dt = time.perf_counter() - t0
    return {"value": n / dt / 1e6, "rows": n, "seconds": dt}


# ---- workloads on the GPU ----------------------------------------------------------------
def run_star(args, kb, W, rt, rank, world, pg, device):
    import torch
    stream = torch.cuda.current_stream()
    fs = args.fact_scale if args.fact_scale is not None else args.scale
    row0, _ = _shard().weak_shard(int(300_000_000 * fs), rank)
    data = W.star(rt, scale=args.scale, fact_row0=row0, fact_scale=fs)
    torch.cuda.synchronize()
    dim_a, dim_b, fact = kb.DeviceBatch(data.dim_a), kb.DeviceBatch(data.dim_b), kb.DeviceBatch(data.fact)

    def make(mode):
        return kb.StarPipeline(rt, kb.star_spec(W.PRED_VALUE, W.PRED_VALUE, group_by=0, mode=mode))

    def timed(pipe, steps, warmup, kernel_events=None, phases=None):
        for _ in range(warmup):
            pipe.reset()
            pipe.build_device(dim_a, dim_b)
            pipe.probe_device(fact)
            pipe.result()
        torch.cuda.synchronize()
        barrier(pg)
        launches0 = rt.launches
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        kev = []
        start.record(stream)
        for _ in range(steps):
            # events between the phases: reset | build | probe | result
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)] if kernel_events is not None else None
            if ev:
                ev[0].record(stream)
            pipe.reset()
            if ev:
                ev[1].record(stream)
            pipe.build_device(dim_a, dim_b)
            if ev:
                ev[2].record(stream)
            pipe.probe_device(fact)
            if ev:
                ev[3].record(stream)
            pipe.result()
            if ev:
                ev[4].record(stream)
                kev.append(ev)
        end.record(stream)
        torch.cuda.synchronize()
        barrier(pg)
        ms = start.elapsed_time(end) / steps
        if kernel_events is not None:
            kernel_events.extend(ev[2].elapsed_time(ev[3]) for ev in kev)
            if phases is not None:
                phases["_steps"] = [ev[0].elapsed_time(ev[4]) for ev in kev]
            if phases is not None:
                for name, i in (("reset", 0), ("build", 1), ("probe", 2), ("result", 3)):
                    phases[name] = statistics.median(ev[i].elapsed_time(ev[i + 1]) for ev in kev)
        return ms, rt.launches - launches0

    fused = make(kb.STAR_FUSED)
    kernel_ms = []
    phases = {}
    with Clocks(device) as clk:
        ms, launches = timed(fused, args.steps, args.warmup, kernel_ms, phases)
    ms_max = max_over_ranks(pg, ms, device)
    step_ms = sorted(phases.pop("_steps"))
    latency = {"p50": max_over_ranks(pg, percentile(step_ms, 50), device),
               "p99": max_over_ranks(pg, percentile(step_ms, 99), device),
               "max": max_over_ranks(pg, step_ms[-1], device), "steps": len(step_ms),
               "what": "whole-query step time (device events), max over ranks"}
    counters = fused.counters()
    result = fused.result()
    # Each rank holds the groups of its own fact rows; the job's answer is
    # their merge (a gather of a few groups per rank).
    partial = {int(g): (float(v), 0) for g, v in zip(result.column(0).to_pylist(), result.column(1).to_pylist())}
    merged = _shard().all_merge_groups(pg, partial) if pg is not None else partial
    plain = make(kb.STAR_PLAIN)
    plain_ms, _ = timed(plain, max(2, args.steps // 2), 1)
    plain_ms = max_over_ranks(pg, plain_ms, device)
    plain_res = plain.result()
    # fused and plain agree (same groups; sums within the float tolerance)
    fr = dict(zip(result.column(0).to_pylist(), result.column(1).to_pylist()))
    pr = dict(zip(plain_res.column(0).to_pylist(), plain_res.column(1).to_pylist()))
    agree = sorted(fr) == sorted(pr) and all(abs(fr[k] - pr[k]) <= 1e-12 * abs(pr[k]) for k in fr)
    nf = data.fact_rows
    # The dominant launch pair: the fact probe (star_scan_kernel streams fk_b
    # and appends the rows passing B's filter; star_join_kernel probes them).
    # Algorithmic bytes per unit: 16 B per fact row (both key columns) and
    # 16 B per joined row (price and discount). The design reads fk_a only in
    # the 32-byte sectors of rows that pass B's filter, counted by the scan;
    # that figure is reported beside it.
    kern_ms = statistics.median(kernel_ms)
    alg_bytes = 16 * nf + 16 * counters["joined_rows"]
    sector_bytes = 8 * nf + 32 * counters["fk_a_sectors"] + 64 * counters["joined_rows"]
    peak, peak_kind = hbm_peak()
    achieved = alg_bytes / (kern_ms * 1e-3) / 1e9
    out = {
        "metric": "star join+agg probe Mrows/s (fact rows per second, whole query)",
        "value": world * nf / (ms_max * 1e-3) / 1e6,
        "unit": "Mrows/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_max,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "int64 keys, float64 sums",
        "data": "synthetic (seeded counter-based generators on the device)",
        "config": star_config(args.scale, fs),
        "mode": "fused (batched) pipeline",
        "groups": len(merged),
        "gpu_launches": launches,
        "latency_ms": latency,
        "phases_ms": phases,
        "roofline": {"bound": "hbm", "kernel": "star_scan_kernel + star_join_kernel (fact probe)",
                     "achieved": achieved, "peak": peak, "peak_source": peak_kind, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": profile_traffic("star_probe", nf),
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the scan + join pair "
                                       "on the 30M-fact-row case (profiles/star_probe_traffic.txt), scaled by fact rows",
                     "algorithmic_bytes_per_launch": alg_bytes, "kernel_ms": kern_ms,
                     "sectors_read_bytes": sector_bytes,
                     "sectors_read_GBps": sector_bytes / (kern_ms * 1e-3) / 1e9},
        "plain": {"ms_per_step": plain_ms, "value": world * nf / (plain_ms * 1e-3) / 1e6,
                  "fused_speedup": plain_ms / ms_max, "results_agree": agree},
        "counters": {k: counters[k] for k in ("passed_filters", "joined_rows", "dim_a_keys", "dim_b_keys",
                                              "filter_a_bytes", "filter_b_bytes", "fk_a_sectors")},
        "clocks": clk.summary(),
    }
    del plain
    host = None
    if not args.no_e2e or (rank == 0 and not args.no_cpu):
        host = HostStar(data)
    if not args.no_e2e:
        out["e2e"] = run_star_e2e(args, kb, W, rt, data, host, pg, device)
    if rank == 0 and not args.no_cpu:
        # The CPU leg: the oracle's star query on the host cores over every
        # fact row of this rank (the same host buffers the e2e leg reads),
        # timed, and its answer checked against the GPU's.
        threads = os.cpu_count() or 1
        kind = _oracle().use_native()
        fact = tuple(h.numpy() for h in host.fact_cols)
        dims = [tuple(h.numpy() for h in cols) for cols in (host.dim_a_cols, host.dim_b_cols)]
        secs, ans = cpu_star_full(fact, dims, threads, runs=3)
        out["cpu_baseline"] = {"value": nf / secs / 1e6, "unit": "Mrows/s", "cores": threads, "kind": "port",
                               "sample": f"the whole query over all {nf} fact rows (no extrapolation), median of 3 "
                                         f"runs; oracle built -O3 ({kind})",
                               "build_s": ans[3], "probe_s": ans[4]}
        out["parity"] = star_parity(fr, counters, ans, nf)
    return out


class HostStar:
    """Page-locked host copies of the star query's columns (Arrow batches
    over them, and the tensors that own the memory)."""

    def __init__(self, data):
        import pyarrow as pa
        import torch

        def host_batch(cols):
            arrays, names, keep = [], [], []
            for name, t, _ in cols:
                h = torch.empty(t.shape, dtype=t.dtype, pin_memory=True)
                h.copy_(t)
                keep.append(h)
                arrays.append(pa.array(h.numpy()))
                names.append(name)
            return pa.RecordBatch.from_arrays(arrays, names=names), keep

        self.fact, self.fact_cols = host_batch(data.fact)
        self.dim_a, self.dim_a_cols = host_batch(data.dim_a)
        self.dim_b, self.dim_b_cols = host_batch(data.dim_b)


def percentile(sorted_values, q):
    """The q-th percentile (nearest rank) of an ascending list."""
    if not sorted_values:
        return None
    i = min(len(sorted_values) - 1, max(0, int(round(q / 100.0 * len(sorted_values) + 0.5)) - 1))
    return sorted_values[i]


def run_star_e2e(args, kb, W, rt, data, host, pg, device):
    """The same query through the C ABI with host (pinned) Arrow buffers; the
    host-to-device copies and the result's device-to-host read are timed."""
    import torch

    fact, dim_a, dim_b = host.fact, host.dim_a, host.dim_b
    pipe = kb.StarPipeline(rt, kb.star_spec(W.PRED_VALUE, W.PRED_VALUE, group_by=0, mode=kb.STAR_FUSED))
    steps = max(2, args.steps // 2)
    for _ in range(args.warmup):
        pipe.reset()
        pipe.build(dim_a, dim_b)
        pipe.probe(fact)
        pipe.result()
    torch.cuda.synchronize()
    barrier(pg)
    t0 = time.perf_counter()
    ph = {"build": [], "probe": [], "result": []}
    for _ in range(steps):
        pipe.reset()
        a = time.perf_counter()
        pipe.build(dim_a, dim_b)
        b = time.perf_counter()
        pipe.probe(fact)
        c = time.perf_counter()
        res = pipe.result()
        ph["build"].append(b - a)
        ph["probe"].append(c - b)
        ph["result"].append(time.perf_counter() - c)
    torch.cuda.synchronize()
    dt = (time.perf_counter() - t0) / steps
    dt = max_over_ranks(pg, dt, device)
    world = int(os.environ.get("WORLD_SIZE", "1"))
    c = pipe.counters()
    # The host columns are page-locked: fk_b of every fact row crosses the
    # host link in bulk copies; the kernels read the rest in place, so every
    # dimension row (key, pred, attr), the fk_a sectors of rows that passed
    # B's filter and the price and discount sectors of joined rows cross it;
    # nothing else does.
    dims = sum(t.numel() * t.element_size() for _, t, _ in data.dim_a + data.dim_b)
    h2d = dims + 8 * data.fact_rows + 32 * c["fk_a_sectors"] + 64 * c["joined_rows"]
    resident = sum(t.numel() * t.element_size() for _, t, _ in data.fact + data.dim_a + data.dim_b)
    return {"value": world * data.fact_rows / dt / 1e6, "unit": "Mrows/s", "h2d_bytes_per_step": h2d,
            "d2h_bytes_per_step": res.num_rows * 12, "ms_per_step": dt * 1e3, "steps": steps,
            "host_input_bytes": resident,
            "phases_ms": {k: statistics.median(v) * 1e3 for k, v in ph.items()},
            "transfer": "page-locked host Arrow buffers: fk_b (read whole) in bulk copies of 64 MiB into HBM on a "
                        "copy stream, three in flight, overlapping the kernels; dimension columns, fk_a, price "
                        "and discount read in place by the kernels (h2d counts their 32-byte sectors)",
            "timing": "host wall clock around synchronous C-ABI calls"}


SWEEP_LOADS = (0.25, 0.5, 1.0, 1.5)


def run_serve(args, kb, W, rt, rank, world, pg, device):
    """The served request stream: join + grouped aggregate requests against
    resident tables, batched (ticks over a device work queue) against plain
    (one request at a time through the operators). Closed loop (every request
    queued at once) gives each mode's capacity; open loop (Poisson arrivals)
    at equal offered loads gives p50 / p99 latency."""
    import numpy as np
    import torch
    temps = W.serve_templates(rt, args.templates, scale=args.scale)
    torch.cuda.synchronize()
    tables_b = [kb.DeviceBatch(t.build) for t in temps]
    probes = [kb.DeviceBatch(t.probe) for t in temps]
    rows_of = np.array([t.probe_rows for t in temps], dtype=np.float64)

    def server(mode):
        s = kb.Server(rt, kb.server_options(mode=mode, tick_rows=args.tick_rows,
                                            hbm_budget_bytes=args.serve_budget))
        tids = [s.add_table(tb) for tb in tables_b]
        torch.cuda.synchronize()
        return s, tids

    def stream(mode, arrivals, which, warm=0):
        s, tids = server(mode)
        for j in range(min(warm, len(temps))):  # warm the tables and the tuner
            s.submit(tids[j], probes[j])
        while s.step(wait=True) > 0 or s.poll() is not None:
            while s.poll() is not None:
                pass
        n = len(arrivals)
        done = np.full(n, np.nan)
        ids = {}
        i = 0
        t0 = time.perf_counter()
        finished = 0
        while finished < n:
            now = time.perf_counter() - t0
            while i < n and arrivals[i] <= now:
                ids[s.submit(tids[which[i]], probes[which[i]])] = i
                i += 1
            left = s.step(wait=False)
            while True:
                p = s.poll()
                if p is None:
                    break
                rid, st, _ = p
                if st != kb.OK:
                    raise RuntimeError(f"request failed with status {st}")
                done[ids.pop(rid)] = time.perf_counter() - t0
                finished += 1
            if left == 0 and i < n:
                time.sleep(max(0.0, min(arrivals[i] - (time.perf_counter() - t0), 0.001)))
        elapsed = np.nanmax(done) - arrivals[0]
        lat = (done - arrivals) * 1e3
        stats = s.stats()
        s.close()
        return {"requests": n, "elapsed_s": float(elapsed), "requests_per_s": n / elapsed,
                "Mrows_per_s": float(rows_of[which].sum() / elapsed / 1e6),
                "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)), "stats": stats}

    n = args.requests
    zero, which = W.serve_arrivals(n, 0.0, len(temps))
    zero = np.zeros(n)
    sweep = None
    with Clocks(device) as clk:
        cap_b = stream(kb.SERVE_BATCHED, zero, which, warm=len(temps))
        cap_p = stream(kb.SERVE_PLAIN, zero[: args.plain_requests], which[: args.plain_requests], warm=2)
        load = args.serve_load
        rate = load * cap_p["requests_per_s"]
        arr, wh = W.serve_arrivals(args.plain_requests, rate, len(temps))
        at_plain_p = stream(kb.SERVE_PLAIN, arr, wh, warm=2)
        at_plain_b = stream(kb.SERVE_BATCHED, arr, wh, warm=len(temps))
        rate_b = load * cap_b["requests_per_s"]
        arr_b, wh_b = W.serve_arrivals(n, rate_b, len(temps))
        at_batched = stream(kb.SERVE_BATCHED, arr_b, wh_b, warm=len(temps))
        if args.serve_sweep:
            # Offered load swept from 0.25x to 1.5x of each mode's measured
            # capacity (Poisson arrivals, the same template mix): requests
            # served per second, p50 / p99 latency at each point.
            sweep = {"loads": list(SWEEP_LOADS), "batched": [], "plain": []}
            for mode, cap, count, key in ((kb.SERVE_BATCHED, cap_b, n, "batched"),
                                          (kb.SERVE_PLAIN, cap_p, args.plain_requests, "plain")):
                for f in SWEEP_LOADS:
                    r = f * cap["requests_per_s"]
                    a_s, w_s = W.serve_arrivals(count, r, len(temps))
                    pt = stream(mode, a_s, w_s, warm=len(temps) if mode == kb.SERVE_BATCHED else 2)
                    pt["offered_requests_per_s"] = r
                    pt["offered_load"] = f
                    pt.pop("stats", None)
                    sweep[key].append(pt)
    # the same request alone and in the mix
    s, tids = server(kb.SERVE_BATCHED)
    j = int(which[0])
    rid = s.submit(tids[j], probes[j])
    while s.step(wait=True) > 0:
        pass
    alone = None
    while (p := s.poll()) is not None:
        alone = {int(a): (int(b), int(c)) for a, b, c in zip(*(t.cpu().tolist() for t in p[2].columns))} if p[2].rows else {}
    mix_ids = [s.submit(tids[int(w)], probes[int(w)]) for w in which[:64]]
    first = mix_ids[0]
    in_mix = None
    while s.step(wait=True) > 0 or in_mix is None:
        while (p := s.poll()) is not None:
            if p[0] == first:
                in_mix = {int(a): (int(b), int(c)) for a, b, c in zip(*(t.cpu().tolist() for t in p[2].columns))} \
                    if p[2].rows else {}
    s.close()
    peak, kind = hbm_peak()
    alg = 16.0 * cap_b["Mrows_per_s"] * 1e6 / 1e9
    return {
        "metric": "served join+agg requests: probe rows/s (closed loop) and p50/p99 latency (open loop)",
        "value": cap_b["Mrows_per_s"], "unit": "Mrows/s", "n_gpus": world, "steps": n, "warmup": len(temps),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic (seeded counter-based generators on the device)",
        "config": {"workload": "SELECT t.g, SUM(p.x), COUNT(*) FROM p JOIN t USING (k) GROUP BY t.g, request stream",
                   "templates": len(temps), "requests": n, "build_rows": f"log-uniform [1e3, {5e7 * args.scale:.0f}]",
                   "probe_rows": "10 x build", "groups": "log-uniform [10, 1e6]", "match": "uniform [0.1, 1.0]",
                   "tick_rows": args.tick_rows, "offered_load": load,
                   "l2": "templates (probe inputs several GB) larger than L2; no flush"},
        "batched_capacity": cap_b, "plain_capacity": cap_p,
        "capacity_ratio": cap_b["requests_per_s"] / cap_p["requests_per_s"],
        "open_loop_at_plain_load": {"requests_per_s_offered": rate, "plain": at_plain_p, "batched": at_plain_b},
        "open_loop_at_batched_load": {"requests_per_s_offered": rate_b, "batched": at_batched},
        "same_alone_and_in_mix": alone == in_mix,
        "load_sweep": sweep,
        "roofline": {"bound": "hbm", "achieved": alg, "peak": peak, "peak_source": kind, "unit": "GB/s",
                     "frac": alg / peak, "traffic": None,
                     "note": "16 B (k, x) per probe row over the closed-loop batched run"},
        "clocks": clk.summary(),
    }


def output_checksum(res):
    """Order-independent checksum of one join output batch (k, p, b1, b2):
    the wrapping sum over rows of a mix of the four values, NULLs mapped to
    distinct constants; and the row count."""
    import torch
    if res.rows == 0:
        return 0, 0
    mult = (0x9E3779B97F4A7C15 - (1 << 64), 0x62A9D9ED799705F5, 0x165667B19E3779F9, 0x27D4EB2F165667C5)
    null = (0x3C6EF372FE94F82B, 0x5851F42D4C957F2D, 0x14057B7EF767814F, 0x2545F4914F6CDD1D)
    acc = None
    for i, c in enumerate(res.columns):
        v = c
        if res.valid[i] is not None:
            bits = res.valid[i][: (res.rows + 7) // 8]
            m = ((bits.unsqueeze(1) >> torch.arange(8, device=c.device, dtype=torch.uint8)) & 1).reshape(-1)[: res.rows]
            v = torch.where(m.bool(), c, torch.full_like(c, null[i]))
        t = (v ^ (v >> 29)) * mult[i]
        acc = t if acc is None else acc ^ t
    return int(acc.sum()) & (2**64 - 1), res.rows


def cpu_grace(scale):
    """The oracle's left outer hash join (single thread) on the partitioned
    join's workload at `scale`: build + probe rows per second."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    W = importlib.import_module("krishiv-engine_b200.workloads")
    nb, np_ = int(500_000_000 * scale), int(2_000_000_000 * scale)
    dom = int(1_000_000_000 * scale)
    seed = W.GRACE_SEED
    bk, bv = O.gen_column(0, seed, 1, nb, lo=0, hi=dom - 1, null_fraction=0.01)
    pk, pv = O.gen_column(0, seed, 11, np_, lo=0, hi=dom - 1, null_fraction=0.01)
    t0 = time.perf_counter()
    O.hash_join(1, [(bk, bv)], [(pk, pv)])
    dt = time.perf_counter() - t0
    return {"value": (nb + np_) / dt / 1e6, "seconds": dt, "build_rows": nb, "probe_rows": np_}


def run_grace(args, kb, W, rt, rank, world, pg, device):
    """The partitioned join workload: left outer join, 500M build rows x 2B probe rows, under
    a 24 GB device budget (a runtime whose allocations are capped), inputs
    resident in HBM, every output batch consumed by a checksum."""
    import torch
    stream = torch.cuda.current_stream()
    build = W.grace_build(rt, scale=args.scale)
    probe = W.grace_probe(rt, scale=args.scale)
    torch.cuda.synchronize()
    nb, np_ = int(build[0][1].shape[0]), int(probe[0][1].shape[0])
    budget = int(args.grace_budget * args.scale) if args.scale < 1 else int(args.grace_budget)
    capped = kb.Runtime(device, budget, stream.cuda_stream)
    bstep, pstep = 32 << 20, 32 << 20
    phases = {}
    step_phases = []

    def batches(cols, n, step):
        for r0 in range(0, n, step):
            m = min(step, n - r0)
            yield kb.DeviceBatch([(nm, t[r0:r0 + m], None if v is None else v[r0 // 8:(r0 + m + 7) // 8 + 1])
                                  for nm, t, v in cols])

    def run_join(partitioned, r):
        spec = kb.join_spec("left_outer", probe_out=[0, 1], build_out=[1, 2], build_rows_hint=nb,
                            max_output_rows=64 << 20, max_load=args.max_load, radix_bits=args.radix_bits)
        j = kb.HashJoin(r, spec, partitioned=partitioned, device_budget=budget if partitioned else 0,
                        probe_filter_bits=args.grace_filter_bits if partitioned else None)
        t = [time.perf_counter()]
        for db in batches(build, nb, bstep):
            j.build_push_device(db)
        j.build_finish()
        torch.cuda.synchronize()
        t.append(time.perf_counter())
        total, rows, nbatches = 0, 0, 0
        calls = []  # host wall time of each probe batch, its output batches consumed (to find stalls)
        for db in batches(probe, np_, pstep):
            c0 = time.perf_counter()
            for res in j.probe_device_all(db):
                c, n = output_checksum(res)
                total, rows, nbatches = (total + c) & (2**64 - 1), rows + n, nbatches + 1
            calls.append((time.perf_counter() - c0) * 1e3)
        torch.cuda.synchronize()
        t.append(time.perf_counter())
        for res in j.finish_device():
            c, n = output_checksum(res)
            total, rows, nbatches = (total + c) & (2**64 - 1), rows + n, nbatches + 1
        torch.cuda.synchronize()
        t.append(time.perf_counter())
        if partitioned:
            slowest = sorted(range(len(calls)), key=lambda i: calls[i])[-5:]
            phases.update(build_s=t[1] - t[0], probe_s=t[2] - t[1], finish_s=t[3] - t[2], output_batches=nbatches,
                          probe_calls=len(calls), probe_call_ms_median=statistics.median(calls) if calls else None,
                          probe_call_ms_slowest={i: round(calls[i], 1) for i in slowest})
            step_phases.append(dict(phases))
        return j, total, rows

    for _ in range(args.warmup):
        run_join(True, capped)
    torch.cuda.synchronize()
    barrier(pg)
    times = []
    launches0 = capped.launches
    with Clocks(device) as clk:
        j = None
        for _ in range(args.steps):
            j = None  # the previous join gives its device and spill memory back first
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            s.record(stream)
            j, total, rows = run_join(True, capped)
            e.record(stream)
            torch.cuda.synchronize()
            times.append((s.elapsed_time(e), (time.perf_counter() - t0) * 1e3))
    ms = max_over_ranks(pg, statistics.median(t for t, _ in times), device)
    counters = j.counters()
    spilled = j.spilled_partitions()
    filtered = j.filtered_probe_rows()
    last_phases = dict(phases)
    launches1 = capped.launches
    del j
    # The unpartitioned join, uncapped, on the same inputs: the same rows.
    _, want_total, want_rows = run_join(False, rt)
    torch.cuda.synchronize()
    peak, kind = hbm_peak()
    alg = 24 * nb + 16 * np_ + 40 * rows
    out = {"metric": "partitioned left outer join under a device budget (build + probe rows per second)",
           "value": world * (nb + np_) / (ms * 1e-3) / 1e6, "unit": "Mrows/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "int64", "data": "synthetic (seeded counter-based generators on the device)",
           "config": {"workload": "left outer join 500M build x 2B probe, 100 heavy probe keys, 1% NULL keys",
                      "build_rows": nb, "probe_rows": np_, "output_rows": rows, "device_budget_bytes": budget,
                      "partitions": counters["partitions"], "spilled_partitions": spilled,
                      "probe_filter_bits_per_key": args.grace_filter_bits, "probe_rows_ruled_out_by_filter": filtered,
                      "consumer": "every output batch read once by an order-independent checksum (timed)",
                      "l2": "inputs (44 GB) larger than L2; no flush"},
           "wall_ms_per_step": statistics.median(w for _, w in times),
           "steps_ms": [round(t, 1) for t, _ in times],
           "phases": dict(last_phases),
           "step_phases": step_phases[-args.steps:],
           "checksum_agrees": (total, rows) == (want_total, want_rows),
           "gpu_launches": (launches1 - launches0) // max(1, args.steps),
           "roofline": {"bound": "hbm", "achieved": alg / (ms * 1e-3) / 1e9, "peak": peak, "peak_source": kind,
                        "unit": "GB/s", "frac": alg / (ms * 1e-3) / 1e9 / peak, "traffic": None,
                        "note": "24 B per build row, 16 B per probe row, 40 B per output row; spilled partitions "
                                "also cross the host link twice"},
           "clocks": clk.summary()}
    if rank == 0 and not args.no_cpu:
        c = cpu_grace(0.001)
        out["cpu_baseline"] = {"value": c["value"], "unit": "Mrows/s", "cores": 1, "kind": "port",
                               "sample": f"the same workload at 1/1000 scale ({c['build_rows']} x {c['probe_rows']} rows)"}
    return out


def run_parquet(args, kb, W, rt, rank, world, pg, device):
    """Parquet column chunks decoded on the device: a file of 64M rows x
    (k int64 in [0, 100K) with 2% NULLs, dictionary encoded; x float64, PLAIN),
    Snappy, row groups of 8M rows, written once to a temporary file. One
    step = every row group's two chunks decoded (their bytes read into
    page-locked host memory beforehand, crossing to the device inside the
    step) with a 5%-of-keys runtime filter evaluated on k's encoded pages.
    The CPU baseline is pyarrow's reader (Arrow C++, all host threads)
    decoding the same columns from the same bytes in memory."""
    import tempfile

    import numpy as np
    import pyarrow as pa
    import pyarrow.parquet as pq
    import torch
    S = importlib.import_module("krishiv-engine_b200.scan")
    n = int(64_000_000 * args.scale)
    rng = np.random.default_rng(5)
    k = rng.integers(0, 100_000, n).astype(np.int64)
    kv = rng.random(n) >= 0.02
    x = rng.random(n)
    table = pa.table({"k": pa.array(k, mask=~kv), "x": x})
    path = os.path.join(tempfile.mkdtemp(), "bench.parquet")
    pq.write_table(table, path, compression=args.parquet_codec, row_group_size=8 << 20, use_dictionary=["k"])
    del table
    md = pq.ParquetFile(path).metadata
    chunks = []
    with open(path, "rb") as f:
        for rg in range(md.num_row_groups):
            for ci, fmt in ((0, "l"), (1, "g")):
                data, d = S.column_chunk(f, md, rg, ci)
                host = torch.empty(len(data), dtype=torch.uint8, pin_memory=True)
                host.numpy()[:] = np.frombuffer(data, dtype=np.uint8)
                chunks.append((host.numpy(), d, fmt, ci == 0))
    encoded = sum(c[0].size for c in chunks)
    build = rng.choice(100_000, 5_000, replace=False).astype(np.int64)
    kf = kb.KeyFilter.build(rt, pa.record_batch([pa.array(build)], names=["k"]), 0)
    stream = torch.cuda.current_stream()

    per_chunk = []  # host wall ms of each call (each call waits for its kernels)

    def step():
        passing, keep = 0, []
        per_chunk.clear()
        for buf, d, fmt, key in chunks:
            t0 = time.perf_counter()
            res, info = kb.parquet_decode_chunk(rt, buf, d["physical_type"], d["codec"], d["max_def_level"],
                                                d["num_values"], fmt, "", kf if key else None)
            per_chunk.append((fmt, info["pages"], round((time.perf_counter() - t0) * 1e3, 2)))
            keep.append(res)
            if key:
                passing += info["passing_rows"]
        return passing, keep

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    launches0 = rt.launches
    times = []
    with Clocks(device) as clk:
        for _ in range(args.steps):
            s_, e_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s_.record(stream)
            passing, keep = step()
            e_.record(stream)
            torch.cuda.synchronize()
            times.append(s_.elapsed_time(e_))
            del keep
    ms = max_over_ranks(pg, statistics.median(times), device)
    # the same filter evaluated on the decoded keys (KeyFilter::evaluate over pyarrow's decode of k)
    import pyarrow.compute as pc
    ev = kf.evaluate(pa.record_batch([pa.array(k, mask=~kv)], names=["k"]), 0)
    want = int(pc.sum(ev).as_py() or 0)
    decoded = n * 8 * 2 + n // 8
    peak, kind = hbm_peak()
    out = {"metric": "Parquet column chunks decoded on the device (rows per second, two columns, filter on the key)",
           "value": world * n / (ms * 1e-3) / 1e6, "unit": "Mrows/s", "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "int64 / float64", "data": "synthetic (seeded numpy, written by pyarrow)",
           "config": {"workload": f"{n} rows x (k int64 dictionary 2% NULLs, x float64 PLAIN), "
                                  f"{args.parquet_codec}, row groups of 8M rows", "encoded_bytes": encoded,
                      "decoded_bytes": decoded,
                      "filter": "5,000 of 100,000 keys, evaluated once per dictionary entry",
                      "transfer": "chunk bytes in page-locked host memory, copied to the device inside the step"},
           "encoded_GBps": encoded / (ms * 1e-3) / 1e9, "decoded_GBps": decoded / (ms * 1e-3) / 1e9,
           "steps_ms": [round(t, 2) for t in times],
           "filter_agrees": passing == want, "passing_rows": passing,
           "calls_ms": [list(c) for c in per_chunk],
           "gpu_launches": (rt.launches - launches0) // max(1, args.steps),
           "roofline": {"bound": "hbm", "achieved": (encoded * 2 + decoded) / (ms * 1e-3) / 1e9, "peak": peak,
                        "peak_source": kind, "unit": "GB/s", "frac": (encoded * 2 + decoded) / (ms * 1e-3) / 1e9 / peak,
                        "traffic": None, "note": "encoded bytes staged (read + write) + decoded column bytes written; "
                                                 "the host-to-device copy of the encoded bytes is inside the step"},
           "clocks": clk.summary()}
    if rank == 0 and not args.no_cpu:
        import pyarrow as pa_
        raw = open(path, "rb").read()
        t = []
        for _ in range(3):
            t0 = time.perf_counter()
            pq.read_table(pa_.BufferReader(raw), columns=["k", "x"], use_threads=True)
            t.append(time.perf_counter() - t0)
        cpu_ms = statistics.median(t) * 1e3
        out["cpu_baseline"] = {"value": n / (cpu_ms * 1e-3) / 1e6, "unit": "Mrows/s", "cores": os.cpu_count(),
                               "kind": "pyarrow", "sample": "pyarrow 24 (Arrow C++) read_table of the same two columns "
                                                          "from the file's bytes in memory, all host threads, median of 3"}
    os.remove(path)
    os.rmdir(os.path.dirname(path))
    return out


def profile_traffic(name, rows):
    """DRAM bytes (read + write) of one launch of `name` over `rows` fact
    rows, from the committed ncu summary profiles/<name>_traffic.txt (line
    'dram_bytes_per_fact_row: X'), scaled to `rows`."""
    path = os.path.join(ROOT, "profiles", f"{name}_traffic.txt")
    try:
        for line in open(path):
            if line.startswith("dram_bytes_per_fact_row:"):
                return float(line.split(":")[1]) * rows
    except OSError:
        pass
    return None


def run_join(args, kb, W, rt, rank, world, pg, device):
    import torch
    stream = torch.cuda.current_stream()
    build, probe = W.join(rt, scale=args.scale)
    torch.cuda.synchronize()
    bb, pb = kb.DeviceBatch(build), kb.DeviceBatch(probe)
    nb, np_ = int(build[0][1].shape[0]), int(probe[0][1].shape[0])

    phase = {"build": [], "probe": []}

    def step(ev=None):
        j = kb.HashJoin(rt, kb.join_spec("inner", probe_out=[0, 1], build_out=[1], build_rows_hint=nb,
                                         max_load=args.max_load))
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)] if ev is not None else None
        if e:
            e[0].record(stream)
        j.build_push_device(bb)
        j.build_finish()
        if e:
            e[1].record(stream)
        r = j.probe_device(pb)
        if e:
            e[2].record(stream)
            ev.append(e)
        return j, r

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier(pg)
    launches0 = rt.launches
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    evs = []
    with Clocks(device) as clk:
        s.record(stream)
        for _ in range(args.steps):
            j, r = step(evs)
        e.record(stream)
        torch.cuda.synchronize()
    ms = max_over_ranks(pg, s.elapsed_time(e) / args.steps, device)
    phase["build"] = statistics.median(x[0].elapsed_time(x[1]) for x in evs)
    phase["probe"] = statistics.median(x[1].elapsed_time(x[2]) for x in evs)
    out_rows = r.rows
    alg = 16 * nb + 12 * np_ + 20 * out_rows
    peak, kind = hbm_peak()
    return {"metric": "plain inner hash join (build+probe rows per second)",
            "value": world * (nb + np_) / (ms * 1e-3) / 1e6, "unit": "Mrows/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64 keys", "data": "synthetic",
            "config": {"workload": "inner join 1M build x 10M probe (50% match), output (k, v, w)",
                       "max_load": args.max_load or 0.5,
                       "build_rows": nb, "probe_rows": np_, "output_rows": out_rows,
                       "l2": "inputs (136 MB) larger than L2; each step rebuilds the table"},
            "gpu_launches": rt.launches - launches0,
            "phases_ms": phase,
            "roofline": {"bound": "hbm", "achieved": alg / (ms * 1e-3) / 1e9, "peak": peak, "peak_source": kind,
                         "unit": "GB/s", "frac": alg / (ms * 1e-3) / 1e9 / peak, "traffic": None,
                         "note": "whole step (build + probe); 16 B per build row, 12 B per probe row, 20 B per output row"},
            "clocks": clk.summary(),
            "cpu_baseline": None if args.no_cpu or rank != 0 else dict(
                unit="Mrows/s", cores=1, kind="port", sample="the whole workload", **{
                    k: v for k, v in cpu_join(args.scale).items() if k == "value"})}


def run_agg(args, kb, W, rt, rank, world, pg, device):
    import torch
    stream = torch.cuda.current_stream()
    cols = W.agg(rt, scale=args.scale)
    torch.cuda.synchronize()
    db = kb.DeviceBatch(cols)
    n = int(cols[0][1].shape[0])
    aggs = [(f, c) for c in (1, 2, 3) for f in ("sum", "count", "min", "max", "avg")]

    phase_ev = []
    host = {"create": [], "push": [], "finish": [], "result": [], "release": []}  # host wall ms per call

    def step(mode, ev=None):
        h = [time.perf_counter()]
        a = kb.HashAggregate(rt, kb.agg_spec(0, aggs, mode=mode, expected_groups=1_000_000))
        h.append(time.perf_counter())
        e = [torch.cuda.Event(enable_timing=True) for _ in range(3)] if ev is not None else None
        if e:
            e[0].record(stream)
        a.push_device(db)
        h.append(time.perf_counter())
        a.finish()
        h.append(time.perf_counter())
        if e:
            e[1].record(stream)
        r = a.result_device()
        if e:
            e[2].record(stream)
            ev.append(e)
        h.append(time.perf_counter())
        del a
        h.append(time.perf_counter())
        if ev is not None:
            for k, t0, t1 in zip(host, h, h[1:]):
                host[k].append((t1 - t0) * 1e3)
        return r

    res, clocks = {}, {}
    for mode, name in ((kb.MODE_SHARED, "shared"), (kb.MODE_GLOBAL, "global")):
        for _ in range(args.warmup):
            step(mode)
        torch.cuda.synchronize()
        barrier(pg)
        launches0 = rt.launches
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with Clocks(device) as clk:
            s.record(stream)
            for _ in range(args.steps):
                r = step(mode, phase_ev if name == "shared" else None)
            e.record(stream)
            torch.cuda.synchronize()
        clocks[name] = clk.summary()
        res[name] = (max_over_ranks(pg, s.elapsed_time(e) / args.steps, device), rt.launches - launches0, r.rows)
    ms, launches, groups = res["shared"]
    alg = n * (8 + 8 + 8 + 4 + 3 / 8) + groups * 136
    peak, kind = hbm_peak()
    return {"metric": "grouped aggregate rows per second", "value": world * n / (ms * 1e-3) / 1e6, "unit": "Mrows/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int128/double-double",
            "data": "synthetic", "config": {"workload": "100M rows Zipf(1.1) over 1M keys, 15 aggregates",
                                            "rows": n, "groups": groups,
                                            "l2": "inputs (2.8 GB) larger than L2; no flush"},
            "gpu_launches": launches,
            "phases_ms": {"push": statistics.median(x[0].elapsed_time(x[1]) for x in phase_ev),
                          "result": statistics.median(x[1].elapsed_time(x[2]) for x in phase_ev)},
            "host_ms": {k: round(statistics.median(v), 3) for k, v in host.items() if v},
            "plain_global_table": {"ms_per_step": res["global"][0], "value": world * n / (res["global"][0] * 1e-3) / 1e6},
            "roofline": {"bound": "hbm", "achieved": alg / (ms * 1e-3) / 1e9, "peak": peak, "peak_source": kind,
                         "unit": "GB/s", "frac": alg / (ms * 1e-3) / 1e9 / peak, "traffic": None,
                         "note": "whole step; 28.4 B per row (key, three value columns, three bitmaps) + 136 B per group"},
            "clocks": clocks["shared"],
            "cpu_baseline": None if args.no_cpu or rank != 0 else dict(
                unit="Mrows/s", cores=1, kind="port", sample=f"first {min(args.cpu_sample, n)} rows", **{
                    k: v for k, v in cpu_agg(args.scale, min(args.cpu_sample, n)).items() if k == "value"})}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["star", "join", "agg", "serve", "grace", "parquet"], default="star")
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--fact-scale", type=float, default=None,
                    help="size the fact table alone (profiling small cases with full dimensions)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-sample", type=int, default=20_000_000)
    ap.add_argument("--requests", type=int, default=2000, help="serve: requests per batched run")
    ap.add_argument("--plain-requests", type=int, default=400, help="serve: requests per plain run")
    ap.add_argument("--templates", type=int, default=32, help="serve: request templates")
    ap.add_argument("--tick-rows", type=int, default=16 << 20, help="serve: probe rows per tick")
    ap.add_argument("--serve-budget", type=int, default=8 << 30, help="serve: HBM budget of running requests")
    ap.add_argument("--serve-load", type=float, default=0.7, help="serve: offered load / capacity")
    ap.add_argument("--serve-sweep", action="store_true",
                    help="serve: also sweep the offered load over 0.25x..1.5x of each mode's capacity")
    ap.add_argument("--grace-budget", type=int, default=24 << 30, help="grace: device budget of the join")
    ap.add_argument("--max-load", type=float, default=0.0, help="join, grace: hash table load factor (0: default)")
    ap.add_argument("--radix-bits", type=int, default=0, help="grace: level-0 partition bits (0: chosen)")
    ap.add_argument("--parquet-codec", default="SNAPPY", choices=["SNAPPY", "NONE"],
                    help="parquet: the file's compression codec")
    ap.add_argument("--grace-filter-bits", type=int, default=10,
                    help="grace: bits per build key of the partition pass's Bloom filter (0: none)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    threads = os.cpu_count() or 1

    if args.impl == "reference":
        # The reference's CPU operators on the host cores: rank 0 alone works
        # (no process group; the other ranks exit at once).
        if int(os.environ.get("RANK", "0")) != 0:
            return
        O = _oracle()
        kind = O.use_native()
        fs = args.fact_scale if args.fact_scale is not None else args.scale
        nf = int(300_000_000 * fs)
        inputs = cpu_star_inputs(args.scale, fs, threads)
        if inputs is not None:
            fact, dims = inputs
            # each step: the whole query over every fact row (no extrapolation)
            secs, _ = cpu_star_full(fact, dims, threads, runs=args.warmup)
            times = []
            for _ in range(args.steps):
                t, _ = cpu_star_full(fact, dims, threads, runs=1)
                times.append(t)
            v = nf / statistics.median(times) / 1e6
            sample = (f"the whole query over all {nf} fact rows per step (dimension builds, key filters, probe, "
                      f"grouped sums; no extrapolation); median of {args.steps} steps; oracle built -O3 ({kind})")
        else:
            steps = []
            info = None
            for _ in range(args.warmup + args.steps):
                info = cpu_star(args.scale, min(args.cpu_sample, 5_000_000), threads)
                steps.append(info["value"])
            v = statistics.median(steps[args.warmup:])
            sample = (f"full dimensions, first {info['sample_rows']} fact rows per step, whole-query rate "
                      f"extrapolated (build + full probe): too little free host memory for all {nf} rows")
        line = {"impl": "reference", "metric": "star join+agg probe Mrows/s (fact rows per second, whole query)",
                "value": v, "unit": "Mrows/s", "n_gpus": args.gpus, "device": "host CPU cores", "steps": args.steps,
                "warmup": args.warmup, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "config": star_config(args.scale, fs),
                "cpu_baseline": {"value": v, "unit": "Mrows/s", "cores": threads, "kind": "port", "sample": sample},
                "e2e": {"value": v, "unit": "Mrows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    rank, world, local, pg = dist_init(args.gpus)
    import torch
    torch.cuda.set_device(local)
    device = local
    kb = importlib.import_module("krishiv-engine_b200")
    W = importlib.import_module("krishiv-engine_b200.workloads")
    rt = kb.Runtime.on_torch_stream(local)
    runner = {"star": run_star, "join": run_join, "agg": run_agg, "serve": run_serve, "grace": run_grace,
              "parquet": run_parquet}[args.workload]
    out = runner(args, kb, W, rt, rank, world, pg, device)
    if rank == 0:
        print(json.dumps(out))
    if pg is not None:
        pg.destroy_process_group()


if __name__ == "__main__":
    main()
