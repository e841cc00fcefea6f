"""Benchmark: KushDB hot-path query throughput on B200.

Workload (default): the Q1-shape group-by at 6,000,000 rows -- ScanSelect
(date <= 10471) -> GroupByAggregate (2 enum keys, 8 aggregates) -> OrderBy --
on seeded synthetic columns (the TPC-H dataset the reference uses is not
available).  Metric: rows/s (whole job), with the roofline of the dominant
kernel against the measured HBM copy bandwidth.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload group_by|scan_agg|join_group|join_group_zipf|batched|serving|skinner|op_hash_join]
                    [--kernel-breakdown]   (skinner: device time per kernel role)

A step is one execution of the query over the resident table.  The timed
region covers exactly K steps on the engine's CUDA stream (events), bracketed
by a barrier and device synchronisation; multi-GPU runs are independent
replicas (weak scaling, max time over ranks).  `--impl reference` times the
CPU implementation of the path (the compiled restatement of the reference's
generated loops and runtime tables, rows split over every host core) on the
same workload, with the host caches evicted between its timed runs as the
GPU's L2 is between GPU steps.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

from kushdb_b200 import workloads as wl  # noqa: E402

L2_BYTES = 126 * 1024 * 1024


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch of
# each workload's dominant kernel at the default size, from one ncu capture
# of the current kernels; other sizes scale it by the rows processed, the
# traffic being proportional to them.
MEASURED_TRAFFIC = {"group_by": 264_039_168 + 3_074_816,
                    "join_group": 126_673_152 + 3_196_672,
                    "scan_agg": 20_026_112}


def make_workload(name: str, scale: float = 1.0):
    """Returns (tables, plan, rows per step, algorithmic bytes per step,
    dominant kernel tag, config dict)."""
    if name == "scan_agg":
        rows = int(1_000_000 * scale)
        t = wl.scan_agg_table(rows=rows)
        cfg = {"workload": "scan_select+aggregate", "rows": rows,
               "predicate": "date<9300 AND discount BETWEEN 0.05 AND 0.07",
               "output": "SUM(price*discount), COUNT(*)"}
        return [t], wl.scan_agg_plan(t), rows, rows * wl.SCAN_AGG_BYTES_PER_ROW, "aggregate", cfg
    if name == "group_by":
        rows = int(6_000_000 * scale)
        t = wl.group_by_table(rows=rows)
        cfg = {"workload": "scan_select+group_by_aggregate+order_by (Q1 shape)", "rows": rows,
               "groups": 4, "aggregates": 8, "predicate": "date<=10471"}
        return [t], wl.group_by_plan(t), rows, rows * wl.GROUP_BY_BYTES_PER_ROW, "group by", cfg
    if name in ("join_group", "join_group_zipf"):
        b_rows, p_rows = int(1_500_000 * scale), int(6_000_000 * scale)
        zipf = name == "join_group_zipf"
        b, p = wl.join_tables(build_rows=b_rows, probe_rows=p_rows, zipf=zipf)
        cfg = {"workload": "hash_join+group_by+order_by (Q3 shape)", "build_rows": b_rows,
               "probe_rows": p_rows, "fk": "zipf s=1.0" if zipf else "uniform"}
        # groups ~ build rows passing the filters (45.7% x 20%); the dominant
        # kernel is the probe pipeline that aggregates into the groups: it
        # reads the probe columns (20 B/row) and writes 16 B per group
        groups = int(b_rows * 0.457 * 0.2)
        cfg["query_algorithmic_bytes"] = wl.join_bytes(b_rows, p_rows, groups)
        return [b, p], wl.join_plan(b, p), b_rows + p_rows, p_rows * 20 + groups * 16, "group by", cfg
    raise SystemExit(f"unknown workload {name}")


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = os.path.join("/tmp", f"kdb_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                smax = float(parts[1])
            except ValueError:
                continue
            for n, v in zip(names, parts[3:7]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def _ranks(values):
    order = sorted(range(len(values)), key=lambda k: values[k])
    r = [0] * len(values)
    for i, k in enumerate(order):
        r[k] = i
    return r


def _host_llc_bytes() -> int:
    """Largest CPU cache the host reports (sysfs), 0 when unknown."""
    best = 0
    base = "/sys/devices/system/cpu/cpu0/cache"
    try:
        for idx in os.listdir(base):
            try:
                with open(os.path.join(base, idx, "size")) as f:
                    txt = f.read().strip().upper()
                mult = 1 << 20 if txt.endswith("M") else (1 << 10 if txt.endswith("K") else 1)
                best = max(best, int(txt.rstrip("KMG")) * mult)
            except (OSError, ValueError):
                continue
    except OSError:
        pass
    return best


class HostCacheFlush:
    """Evicts the host caches between timed CPU steps (a write larger than
    the last-level cache), as the GPU's L2 is flushed between GPU steps:
    repeating a query over the same table would otherwise leave much of a
    264 MB table in a large host cache and time warm reads."""

    def __init__(self):
        self.buf = np.zeros(max(1 << 30, 4 * _host_llc_bytes()), dtype=np.uint8)
        self.k = 0

    def __call__(self):
        self.k = (self.k + 1) & 0xff
        self.buf.fill(self.k)


def run_cpu_baseline(name: str, tables, threads: int = 1):
    """One execution of the compiled CPU baseline loop for the workload
    (oracle/baseline.cc: the reference's generated-code loop + runtime
    structures, restated; one thread like the reference executor, or the rows
    split over `threads` host threads with partial tables merged).  Returns
    seconds."""
    import oracle
    from kushdb_b200.plan import EPOCH_JDN
    if name == "scan_agg":
        return oracle.baseline_scan_agg(tables[0], 9300 + EPOCH_JDN, 0.05, 0.07, threads=threads)[0]
    if name == "group_by":
        return oracle.baseline_group_by(tables[0], 10471 + EPOCH_JDN, _ranks(wl.RF_VALUES),
                                        _ranks(wl.LS_VALUES), threads=threads)[0]
    return oracle.baseline_join_group(tables[0], tables[1], 9204 + EPOCH_JDN,
                                      wl.SEG_VALUES.index("BUILDING"), threads=threads)[0]


def cpu_baseline(name: str, tables, rows: int, repeats: int = 3):
    """Times the compiled CPU baseline on the full workload (a few seconds of
    CPU work at most), on every host core and on one; rows/s from the best
    of `repeats`."""
    import oracle
    threads = oracle.host_threads()
    flush = HostCacheFlush()

    def timed(t):
        flush()
        return run_cpu_baseline(name, tables, t)
    secs = min(timed(threads) for _ in range(repeats))
    secs1 = min(timed(1) for _ in range(repeats))
    del flush
    return rows / secs, {"rows": rows, "seconds": secs, "repeats": repeats, "threads": threads,
                         "single_thread_rows_per_second": rows / secs1}


def run_reference(args):
    """The CPU arm: the reference's path restated (no build of the reference
    is possible here), on all host cores, on the same workload and metric."""
    import oracle
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    threads = oracle.host_threads()
    tables, plan, rows, _, _, cfg = make_workload(args.workload)
    flush = HostCacheFlush()
    for _ in range(args.warmup):
        run_cpu_baseline(args.workload, tables, threads)
    total = 0.0
    for _ in range(args.steps):
        flush()  # outside the timed region (the loop times itself)
        total += run_cpu_baseline(args.workload, tables, threads)
    value = rows * args.steps / total
    line = {
        "impl": "reference", "metric": "rows_per_second", "value": value, "unit": "rows/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total / args.steps * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
        "cpu_baseline": {"value": value, "unit": "rows/s", "cores": threads, "kind": "port",
                         "sample": f"the full {args.workload} workload ({rows} rows) per step: "
                                   "compiled restatement of the reference's generated loop and "
                                   f"runtime tables, rows split over {threads} host threads "
                                   "(partial tables merged); host caches evicted between steps "
                                   f"({flush.buf.nbytes >> 20} MiB write), as the GPU's L2 is"},
        "e2e": {"value": value, "unit": "rows/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


def run_batched(args):
    """Batched form: N uneven join + group-by queries as one captured CUDA
    graph vs the same N queries one at a time through the plain executor."""
    import torch
    from kushdb_b200.engine import Batch, Engine
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    qs = wl.batch_tables(n_queries=args.batch_queries, max_fact=args.batch_max_fact)
    eng = Engine(local)
    for d, f, _, _ in qs:
        eng.register_table(d)
        eng.register_table(f)
    rows = sum(d.rows + f.rows for d, f, _, _ in qs)
    algo_bytes = sum(d.rows * 12 + f.rows * 20 for d, f, _, _ in qs)
    plans = [wl.batch_plan(*q).to_json().encode() for q in qs]
    for p in plans:  # compile + warm the plain pipelines
        eng.execute(p, fetch=False)
    stream = torch.cuda.ExternalStream(eng.stream_handle())
    plain_ms = []
    for _ in range(max(1, args.steps // 5)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for p in plans:
            eng.execute(p, fetch=False)
        e1.record(stream)
        e1.synchronize()
        plain_ms.append(e0.elapsed_time(e1))
    b = Batch(eng, [wl.batch_query_desc(*q) for q in qs])
    report = b.tune(reps=2)
    cfg = b.config()
    b.run()
    launches0 = eng.kernel_launches()
    with ClockSampler(local) as clocks:
        for _ in range(args.warmup):
            b.run_timed(1)
        batch_ms = b.run_timed(args.steps)
    launches = eng.kernel_launches() - launches0
    plain = statistics.median(plain_ms)
    peak, peak_kind = _peaks()
    line = {
        "metric": "queries_per_second", "value": len(qs) / (batch_ms / 1e3), "unit": "queries/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": batch_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "batched scan_select+hash_join+group_by template", "queries": len(qs),
                   "fact_rows": "log-uniform [1e4, %d]" % args.batch_max_fact, "dim_rows": "fact/4",
                   "rows": rows, "selectivity": "uniform [1%, 90%]", "tuned": cfg,
                   "l2": "inputs larger than L2"},
        "plain": {"ms_for_all_queries": plain, "queries_per_second": len(qs) / (plain / 1e3)},
        "speedup_vs_plain": plain / batch_ms,
        "roofline": {"bound": "hbm", "achieved": algo_bytes / (batch_ms / 1e3) / 1e9, "peak": peak,
                     "unit": "GB/s", "frac": algo_bytes / (batch_ms / 1e3) / 1e9 / peak, "traffic": None,
                     "kernel": "whole batch graph", "algorithmic_bytes": algo_bytes,
                     "peak_source": f"{peak_kind} hbm_gbs"},
        "autotune": sorted(report, key=lambda r: r["ms"])[:5],
        "gpu_launches": launches,
        "clocks": clocks.summary(),
    }
    print(json.dumps(line))


def skinner_queries(seed0: int, count: int, min_rows: int = 10_000, max_rows: int = 3_000_000):
    """JOB-style multiway joins: star and chain shapes of 6-8 tables with
    log-uniform sizes, Zipf 0 / 1.5 foreign keys and LIKE '%tok%' filters."""
    out = []
    for i in range(count):
        shape = "star" if i % 2 == 0 else "chain"
        n_tables = 6 + i % 3
        zipf = 1.5 if i % 4 >= 2 else 0.0
        tables, tokens = wl.skinner_tables(shape, n_tables, min_rows=min_rows, max_rows=max_rows, zipf_s=zipf,
                                           seed=seed0 + 31 * i, prefix=f"sk{seed0}_{i}_")
        out.append((f"{shape}{n_tables}{'z' if zipf else ''}", tables, wl.skinner_plan(tables, tokens, shape)))
    return out


def train_join_prior(eng, budget: int, count: int = 16, max_rows: int = 300_000):
    """Trains the learned join-order prior on queries disjoint from the
    measured ones (random-order episodes of smaller instances)."""
    from kushdb_b200.join_prior import fit_prior
    train_q = skinner_queries(7000, count, max_rows=max_rows)
    for _, tables, _ in train_q:
        for t in tables:
            eng.register_table(t)
    t0 = time.perf_counter()
    model, info = fit_prior(eng, [p for _, _, p in train_q], budget, seeds=(0, 1), steps=1500)
    info["seconds"] = time.perf_counter() - t0
    for _, tables, _ in train_q:
        for t in tables:
            eng.drop_table(t.name)
    return model, info


def run_skinner(args):
    """Skinner multiway joins (C5 shapes) one at a time: device time,
    episodes and tuples examined per query under plain UCT and under UCT
    seeded by the learned prior, on the same resident tables."""
    import torch
    from kushdb_b200.engine import Engine
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    eng = Engine(local)
    budget = args.skinner_budget
    model, info = train_join_prior(eng, budget)
    queries = skinner_queries(100, args.skinner_queries)
    for _, tables, _ in queries:
        for t in tables:
            eng.register_table(t)
    stream = torch.cuda.ExternalStream(eng.stream_handle())
    per = {}
    launches0 = eng.kernel_launches()
    with ClockSampler(local) as clocks:
        for policy in ("uct", "prior"):
            eng.set_skinner_policy(policy, prior=model if policy == "prior" else None)
            rows = []
            for name, tables, plan in queries:
                p = plan.to_json().encode()
                eng.set_skinner(budget, 0)
                for _ in range(args.warmup):
                    eng.execute(p, fetch=False)
                ms, eps, work = [], [], []
                for s in range(args.steps):
                    eng.set_skinner(budget, s)
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    n = eng.execute(p, fetch=False)
                    e1.record(stream)
                    e1.synchronize()
                    ms.append(e0.elapsed_time(e1))
                    eps.append(eng.last_skinner_episodes())
                    work.append(eng.last_skinner_work())
                rows.append({"query": name, "tables": len(tables), "rows": sum(t.rows for t in tables),
                             "result_rows": int(n), "ms": statistics.median(ms),
                             "episodes": statistics.median(eps), "work": statistics.median(work)})
            per[policy] = rows
    eng.set_skinner_policy("uct")
    timed_launches = eng.kernel_launches() - launches0
    breakdown = None
    if args.kernel_breakdown:
        # per query (plain UCT): device time by kernel role, from CUDA events
        # around every launch (profiling mode: one fresh execution each)
        breakdown = {}
        eng.set_skinner(budget, 0)
        for name, _, plan in queries:
            eng.set_profiling(True)
            eng.execute(plan.to_json().encode(), fetch=False)
            ks = eng.last_kernels()
            eng.set_profiling(False)
            tags = {}
            for k in ks:
                t = tags.setdefault(k["tag"], [0, 0.0])
                t[0] += 1
                t[1] += k["ms"]
            breakdown[name] = {k: {"launches": v[0], "ms": round(v[1], 4)}
                               for k, v in sorted(tags.items(), key=lambda kv: -kv[1][1])}
    total = {k: sum(r["ms"] for r in v) for k, v in per.items()}
    best = min(total, key=total.get)
    nq = len(queries)
    line = {
        "metric": "queries_per_second", "value": nq / (total[best] / 1e3), "unit": "queries/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": total[best] / nq,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic",
        "config": {"workload": "skinner multiway joins (star/chain, 6-8 tables, rows log-uniform "
                               "[1e4, 3e6], zipf 0/1.5, LIKE '%tok%' filters), one at a time",
                   "queries": nq, "budget_per_episode": budget, "policy": best,
                   "l2": "inputs larger than L2 (126 MB)"},
        "policies": {k: {"ms_total": total[k], "episodes_total": sum(r["episodes"] for r in v),
                         "work_total": sum(r["work"] for r in v)} for k, v in per.items()},
        "prior_training": info,
        "per_query": per,
        "kernel_breakdown_ms": breakdown,
        "gpu_launches": timed_launches,
        "clocks": clocks.summary(),
    }
    print(json.dumps(line))


def run_serving(args):
    """Serving form (C5): requests arrive (all at once, then as a Poisson
    process) and the server's slots run them concurrently.  The default mix
    is Skinner multiway joins (star/chain, 6-8 tables, 1e4-3e6 rows, Zipf
    0/1.5, LIKE filters) under plain UCT and under UCT seeded by the learned
    prior; `--serving-mix mixed` adds scan + aggregate, group-by and join +
    group-by shapes.  Reports queries/s and submission-to-completion
    latency p50/p99, beside the same requests run one at a time."""
    import random
    import torch
    from kushdb_b200.engine import Engine, Server
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    eng = Engine(local)
    budget = args.skinner_budget
    model, info = train_join_prior(eng, budget)
    plans = []
    for name, tables, plan in skinner_queries(100, args.skinner_queries):
        for t in tables:
            eng.register_table(t)
        plans.append((name, plan.to_json().encode()))
    if args.serving_mix == "mixed":
        sa = wl.scan_agg_table(1_000_000, name="srv_sales")
        gb = wl.group_by_table(6_000_000, name="srv_lineitem")
        build, probe = wl.join_tables(1_500_000, 6_000_000)
        for t in (sa, gb, build, probe):
            eng.register_table(t)
        plans += [("scan_agg", wl.scan_agg_plan(sa, date_lt=d).to_json().encode()) for d in (9000, 9800)]
        plans += [("group_by", wl.group_by_plan(gb, date_leq=d).to_json().encode()) for d in (10000, 10471)]
        plans += [("join_group", wl.join_plan(build, probe, date_lt=d).to_json().encode()) for d in (9000, 9204)]
    eng.set_skinner(budget, 0)
    rnd = random.Random(1234)
    n = args.serving_requests
    seq = [plans[rnd.randrange(len(plans))] for _ in range(n)]
    stream = torch.cuda.ExternalStream(eng.stream_handle())
    out = {}
    for policy in ("uct", "prior"):
        eng.set_skinner_policy(policy, prior=model if policy == "prior" else None)
        for _ in range(args.warmup):  # compile and warm every pipeline
            for _, p in plans:
                eng.execute(p, fetch=False)
        # one at a time through the plain API (device time per request)
        alone = {}
        t0 = time.perf_counter()
        for k, p in seq:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            eng.execute(p, fetch=False)
            e1.record(stream)
            e1.synchronize()
            alone.setdefault(k, []).append(e0.elapsed_time(e1))
        seq_s = time.perf_counter() - t0
        res = {"one_at_a_time": {"queries_per_second": n / seq_s,
                                 "device_ms_p50_by_query": {k: statistics.median(v) for k, v in alone.items()}}}
        # all requests at once (saturated), then Poisson arrivals at the fixed
        # rate and at 80% of the saturated throughput (near saturation)
        for mode in ("saturated", "poisson", "poisson_near_saturation"):
            rate = args.serving_rate if mode == "poisson" else \
                0.8 * res.get("saturated", {}).get("queries_per_second", args.serving_rate)
            with ClockSampler(local) as clocks, Server(eng, slots=args.serving_slots,
                                                       hbm_budget_bytes=args.serving_budget_gb << 30) as srv:
                tickets = []
                t0 = time.perf_counter()
                if mode == "saturated":
                    for _, p in seq:
                        tickets.append(srv.submit(p))
                else:
                    gaps = np.random.default_rng(7).exponential(1.0 / rate, n)
                    t_next = t0
                    for (_, p), g in zip(seq, gaps):
                        t_next += g
                        while time.perf_counter() < t_next:
                            pass
                        tickets.append(srv.submit(p))
                for t in tickets:
                    srv.wait(t).close()
                st = srv.stats()
                st["wall_s"] = time.perf_counter() - t0
                if mode != "saturated":
                    st["arrival_rate_qps"] = rate
            st["clocks"] = clocks.summary()
            res[mode] = st
        out[policy] = res
    eng.set_skinner_policy("uct")
    best = max(out, key=lambda k: out[k]["saturated"]["queries_per_second"])
    sat = out[best]["saturated"]
    line = {
        "metric": "queries_per_second", "value": sat["queries_per_second"], "unit": "queries/s",
        "n_gpus": 1, "steps": n, "warmup": args.warmup, "ms_per_step": 1e3 / sat["queries_per_second"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": "served Skinner multiway joins (star/chain, 6-8 tables, rows log-uniform "
                               "[1e4, 3e6], zipf 0/1.5, LIKE '%tok%' filters)"
                               + (" + scan_agg/group_by/join_group" if args.serving_mix == "mixed" else ""),
                   "requests": n, "distinct_queries": len(plans), "slots": args.serving_slots,
                   "hbm_budget_gb": args.serving_budget_gb, "poisson_rate_qps": args.serving_rate,
                   "budget_per_episode": budget, "policy": best, "l2": "inputs larger than L2 (126 MB)"},
        "p50_ms": out[best]["poisson"]["p50_ms"], "p99_ms": out[best]["poisson"]["p99_ms"],
        "near_saturation": {k: out[best]["poisson_near_saturation"].get(k)
                            for k in ("arrival_rate_qps", "queries_per_second", "p50_ms", "p99_ms")},
        "policies": out,
        "speedup_vs_one_at_a_time": sat["queries_per_second"] / out[best]["one_at_a_time"]["queries_per_second"],
        "prior_training": info,
        "gpu_launches": sum(out[k][m]["kernel_launches"] for k in out
                            for m in ("saturated", "poisson", "poisson_near_saturation")),
        "clocks": sat["clocks"],
    }
    print(json.dumps(line))


def run_op_hash_join(args):
    """The per-operator hash join (kdb_hash_build + kdb_hash_probe) on a
    build side larger than L2: 30M unique INT keys, 20M uniform foreign keys
    probed (unordered pairs).  A step builds the table and probes it; the
    kernels' CUDA-event times come from the context's profiling."""
    from kushdb_b200.data import HostColumn, HostTable
    from kushdb_b200.engine import Engine
    from kushdb_b200.operators import HashTable
    from kushdb_b200.plan import Type
    nb, npr = 30_000_000, 20_000_000
    rng = np.random.default_rng(3)
    eng = Engine(0)
    b = HostTable("op_jb")
    b.add(HostColumn("k", Type.Int(), values=(rng.permutation(nb) + 1).astype(np.int32)))
    p = HostTable("op_jp")
    p.add(HostColumn("k", Type.Int(), values=rng.integers(1, nb + 1, npr).astype(np.int32)))
    eng.register_table(b)
    eng.register_table(p)
    eng.set_profiling(True)
    times = {}
    fanout = 0
    with ClockSampler(0) as clocks:
        for step in range(args.warmup + args.steps):
            ht = HashTable(eng, "op_jb", "k", fanout=args.fanout)
            build = eng.last_kernels()
            ht.probe("op_jp", "k", ordered=False)
            probe = eng.last_kernels()
            fanout = ht.info()[0]
            ht.close()
            if step >= args.warmup:
                for x in build + probe:
                    times.setdefault(x["tag"], []).append(x["ms"])
    med = {k: float(np.median(v)) for k, v in times.items()}
    total = sum(med.values())
    line = {"metric": "rows_per_second", "value": (nb + npr) / (total * 1e-3), "unit": "rows/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
            "config": {"workload": "kdb_hash_build + kdb_hash_probe (per-operator)", "build_rows": nb,
                       "probe_rows": npr, "fanout": fanout, "timing": "sum of the kernels' CUDA-event medians"},
            "kernels_ms": med, "clocks": clocks.summary()}
    print(json.dumps(line))
    eng.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="group_by",
                    choices=["group_by", "scan_agg", "join_group", "join_group_zipf", "batched", "serving",
                             "skinner", "op_hash_join"])
    ap.add_argument("--batch-queries", type=int, default=256)
    ap.add_argument("--batch-max-fact", type=int, default=6_000_000)
    ap.add_argument("--rows", type=int, default=0,
                    help="rows per step for scan_agg / group_by / join_group (size sweeps); default: the "
                         "configuration's own size")
    ap.add_argument("--skinner-budget", type=int, default=100_000)
    ap.add_argument("--skinner-queries", type=int, default=8)
    ap.add_argument("--serving-requests", type=int, default=400)
    ap.add_argument("--serving-mix", default="skinner", choices=["skinner", "mixed"])
    ap.add_argument("--serving-slots", type=int, default=16)
    ap.add_argument("--serving-rate", type=float, default=50.0)
    ap.add_argument("--serving-budget-gb", type=int, default=32)
    ap.add_argument("--fanout", type=int, default=0,
                    help="op_hash_join: sub-tables of the build (1 = one table, 0 = automatic)")
    ap.add_argument("--kernel-breakdown", action="store_true",
                    help="skinner: also report each query's device time by kernel role (profiling mode)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-sub", action="store_true",
                    help="only the headline workload (no scan_agg / join_group lines beside group_by)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "batched":
        run_batched(args)
        return
    if args.workload == "serving":
        run_serving(args)
        return
    if args.workload == "skinner":
        run_skinner(args)
        return
    if args.workload == "op_hash_join":
        run_op_hash_join(args)
        return

    import torch
    from kushdb_b200 import replicas
    rank, world, local = replicas.rank_info()
    torch.cuda.set_device(local)
    dist = replicas.init("nccl", timeout_s=300)

    from kushdb_b200.engine import Engine
    eng = Engine(local)
    stream = torch.cuda.ExternalStream(eng.stream_handle())
    scale = 1.0
    if args.rows:
        scale = args.rows / BASE_ROWS[args.workload]
    with ClockSampler(local) as clocks:
        line = measure(args.workload, args, eng, stream, local, world, dist, scale, args.steps, args.warmup,
                       rank == 0)
    line["clocks"] = clocks.summary()
    # the other plain configurations under the same clock: scan + ungrouped
    # aggregate (1M rows) and hash join + group-by (1.5M x 6M, uniform and
    # Zipf s=1.0 foreign keys)
    subs = {}
    if not args.no_sub and args.workload == "group_by" and not args.rows:
        for sub in ("scan_agg", "join_group", "join_group_zipf"):
            subs[sub] = measure(sub, args, eng, stream, local, world, dist, 1.0, args.steps, args.warmup, rank == 0)
    if rank != 0:
        replicas.finish(dist)
        return
    if subs:
        line["sub"] = subs
    print(json.dumps(line))
    replicas.finish(dist)


BASE_ROWS = {"scan_agg": 1_000_000, "group_by": 6_000_000, "join_group": 7_500_000, "join_group_zipf": 7_500_000}


def _gpu_local_cpus(local: int):
    """The host CPUs attached to GPU `local`'s NUMA node (empty when unknown)."""
    try:
        out = subprocess.run(["nvidia-smi", "-i", str(local), "--query-gpu=pci.bus_id", "--format=csv,noheader"],
                             capture_output=True, text=True, timeout=20).stdout.strip().lower()
        bus = out[4:] if out.startswith("0000") and len(out) > 12 else out
        with open(f"/sys/bus/pci/devices/{bus}/local_cpulist") as f:
            spec = f.read().strip()
    except (OSError, subprocess.SubprocessError, ValueError):
        return set()
    cpus = set()
    for part in spec.split(","):
        if "-" in part:
            a, b = part.split("-")
            cpus.update(range(int(a), int(b) + 1))
        elif part:
            cpus.add(int(part))
    return cpus & os.sched_getaffinity(0)


def pin_tables(tables, local: int):
    """Moves every fixed-width column of `tables` into pinned host memory,
    allocated and first touched from the CPUs next to the GPU so that the
    pages sit on the GPU's NUMA node.  Returns the pinned tensors (kept
    alive by the caller) and the bytes per step."""
    import torch
    keep, nbytes = [], 0
    old = os.sched_getaffinity(0)
    near = _gpu_local_cpus(local)
    if near:
        os.sched_setaffinity(0, near)
    try:
        for t in tables:
            for c in t.columns.values():
                for attr in ("values", "nulls"):
                    a = getattr(c, attr)
                    if a is None:
                        continue
                    pt = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
                    pt.numpy()[:] = np.frombuffer(np.ascontiguousarray(a).tobytes(), np.uint8)
                    setattr(c, attr, pt.numpy().view(a.dtype))
                    keep.append(pt)
                    nbytes += a.nbytes
    finally:
        if near:
            os.sched_setaffinity(0, old)
    return keep, nbytes, len(near)


def pinned_copy_gbs(keep, local: int, stream) -> float:
    """The host link's rate in this run: the same pinned buffers copied to
    the device with plain cudaMemcpyAsync, one copy per buffer on one stream
    (median of 5)."""
    import torch
    dev = [torch.empty(k.numel(), dtype=torch.uint8, device=f"cuda:{local}") for k in keep]
    total = sum(k.numel() for k in keep)
    ms = []
    for _ in range(6):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            for d, h in zip(dev, keep):
                d.copy_(h, non_blocking=True)
            e1.record(stream)
        e1.synchronize()
        ms.append(e0.elapsed_time(e1))
    del dev
    return total / (statistics.median(ms[1:]) / 1e3) / 1e9


def measure(name, args, eng, stream, local, world, dist, scale, steps, warmup, with_cpu):
    """One plain workload: device-resident throughput (CUDA events over
    exactly `steps` steps, L2 flushed between steps when the inputs fit in
    it), the dominant kernel's roofline, end to end from pinned host memory
    through kdb_query_execute_host, and the CPU arm."""
    import torch
    from kushdb_b200 import replicas
    tables, plan_tree, rows, algo_bytes, dom_tag, cfg = make_workload(name, scale)
    plan = plan_tree.to_json().encode()  # the statement text, prepared once like a client would
    for t in tables:
        eng.register_table(t)
    for _ in range(warmup):  # compiles the pipelines (cached) and records the prepared query
        eng.execute(plan)
    torch.cuda.synchronize()

    # L2 flush between steps: write a 256 MiB buffer, then read another one,
    # so the timed kernels start with none of their inputs in L2 and with no
    # dirty flush lines left to write back while they run
    flush = None
    if algo_bytes < 2 * L2_BYTES:
        flush = (torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device=f"cuda:{local}"),
                 torch.ones(64 * 1024 * 1024, dtype=torch.int32, device=f"cuda:{local}"))

    def flush_l2():
        if flush is not None:
            with torch.cuda.stream(stream):
                flush[0].fill_(1)
                flush[1].sum()

    replicas.barrier(dist)
    torch.cuda.synchronize()
    launches0 = eng.kernel_launches()
    step_ms = []
    for _ in range(steps):
        flush_l2()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        eng.execute(plan)
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
    torch.cuda.synchronize()
    launches = eng.kernel_launches() - launches0
    total_ms = replicas.max_over_ranks(sum(step_ms), dist, f"cuda:{local}")
    replicas.barrier(dist)
    value = replicas.whole_job_rate(rows, steps, world, total_ms)

    # roofline of the dominant kernel: per-launch CUDA events (profiling mode)
    eng.set_profiling(True)
    kern = []
    for _ in range(5):
        flush_l2()
        eng.execute(plan)
        kern.append(eng.last_kernels())
    eng.set_profiling(False)
    dom = [k["ms"] for ks in kern for k in ks if k["tag"] == dom_tag]
    dom_ms = statistics.median(dom) if dom else None
    peak, peak_kind = _peaks()
    achieved = algo_bytes / (dom_ms / 1e3) / 1e9 if dom_ms else None
    kernels_per_query = {}
    for k in kern[-1]:
        kernels_per_query[k["tag"]] = round(kernels_per_query.get(k["tag"], 0) + k["ms"], 5)
    del flush

    # end to end through the public API: every step brings the tables from
    # pinned host memory (chunked copies on several streams) and runs the
    # query (kdb_query_execute_host); the result comes back to the host
    e2e = None
    if not args.no_e2e:
        keep, h2d, near = pin_tables(tables, local)
        link = pinned_copy_gbs(keep, local, stream)
        torch.cuda.synchronize()
        e2e_ms = []
        d2h = 0
        for i in range(max(3, steps // 2) + 2):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = eng.execute_host(plan, tables)
            e1.record(stream)
            e1.synchronize()
            if i >= 2:
                e2e_ms.append(e0.elapsed_time(e1))
            d2h = sum(8 * r.num_rows + r.num_rows for _ in r.columns)
        e2e_med = replicas.max_over_ranks(statistics.median(e2e_ms), dist, f"cuda:{local}")
        h2d_gbs = h2d / (e2e_med / 1e3) / 1e9
        e2e = {"value": replicas.whole_job_rate(rows, 1, world, e2e_med), "unit": "rows/s",
               "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "ms_per_step": e2e_med,
               "h2d_gbs": h2d_gbs, "pinned_copy_gbs": link, "link_frac": h2d_gbs / link,
               "pinned_numa_local_cpus": near,
               "path": "kdb_query_execute_host: chunked H2D on copy streams, then the query"}
        del keep

    cpu = None
    if with_cpu and not args.no_cpu_baseline:
        try:
            v, info = cpu_baseline(name, tables, rows)
            cpu = {"value": v, "unit": "rows/s", "cores": info["threads"], "kind": "port",
                   "single_thread_value": info["single_thread_rows_per_second"],
                   "sample": f"full workload ({info['rows']} rows), best of {info['repeats']}: "
                             f"{info['seconds']:.4f} s on {info['threads']} host threads; compiled "
                             "restatement of the reference's generated loop + runtime tables "
                             "(oracle/baseline.cc), rows split over the threads; host caches evicted "
                             "before each run"}
        except Exception as ex:  # the oracle is a reported baseline, not the product
            cpu = {"value": None, "unit": "rows/s", "cores": 0, "kind": "port", "sample": f"failed: {ex}"}
    for t in tables:
        eng.drop_table(t.name)

    cfg = dict(cfg)
    cfg["l2"] = "flushed between steps (256 MiB write, then 256 MiB read)" if algo_bytes < 2 * L2_BYTES else \
        "inputs larger than L2 (126 MB)"
    return {
        "metric": "rows_per_second", "value": value, "unit": "rows/s", "n_gpus": world,
        "steps": steps, "warmup": warmup, "ms_per_step": total_ms / steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic", "config": cfg,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": (achieved / peak) if achieved else None,
                     "traffic": (round(MEASURED_TRAFFIC[name] * scale) if name in MEASURED_TRAFFIC else None),
                     "kernel": dom_tag, "kernel_ms": dom_ms, "algorithmic_bytes": algo_bytes,
                     "peak_source": f"{peak_kind} hbm_gbs"},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": launches,
        "kernels_ms_per_query": kernels_per_query,
    }


if __name__ == "__main__":
    main()
