#!/usr/bin/env python
"""Benchmark of the fused filter -> join -> group-by path on B200.

Workload (default, "join_group"): build side 10M rows (pk = permutation of
[0,10M), cat U[0,1000)), probe side 100M rows (fk U[0,12M), qty U[1,100],
price U[1,500)); filter qty > 10, inner join fk = pk, group by cat with
SUM(price), COUNT -- one td_execute of one DAG (teide_b200's single-graph
filter -> join -> group form).  A step is one such query.  Seeded synthetic
data; inputs (2.56 GB) are larger than L2, so no flush is needed between steps.

  value  rows/s of probe rows with both tables resident in HBM (td_gpu_pin)
  e2e    the same query from host tables: every step uploads both tables
         (page-locked host memory) and reads the result back
  roofline  the fused probe + aggregate kernel: algorithmic bytes per launch
         (24 B per probe row: fk, qty, price) / its CUDA-event duration

Other workloads (--workload): "group_radix" (200M rows, Zipf keys over 2^24,
filter v1 > 0, COUNT/SUM/MIN/MAX/AVG), "group_sort" (the same group-by with its
5.9M groups sorted by v1_sum descending: td_sort_op over the group node) and
"readme_group" (10M rows, filter flag == 0, group by region, SUM(amount)).

--impl reference runs Teide's own CPU engine (compiled from its sources into
oracle/_ref/) on a bounded sample of the same workload per step, with every
host thread.
"""
import argparse
import functools
import json
import os
import re
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fused filter/join/group-by rows/s & %HBM peak; served q/s + p99 vs plain"
REF_LIB = os.path.join(ROOT, "oracle", "_ref", "libteide_ref.so")


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(name):
    """Per-launch DRAM bytes from the committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    m = re.search(r"traffic_per_launch_bytes\s*=\s*([0-9.eE+]+)", open(p).read())
    return float(m.group(1)) if m else None


class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
             "clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) == 7:
                self.rows.append((time.monotonic(), parts))

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self, t0, t1):
        """Samples taken while [t0, t1] ran (the sampler ticks every 200 ms,
        so a short timed region also takes the ticks just around it)."""
        near = [r for t, r in self.rows if t0 - 0.25 <= t <= t1 + 0.25]
        if not near and self.rows:
            near = [r for _, r in sorted(self.rows, key=lambda x: abs(x[0] - (t0 + t1) / 2))[:3]]
        if not near:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[0]) for r in near if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in near if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in near for i in range(4) if r[3 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(near)}


# ---- workloads through the td.h API ------------------------------------------------

def workload_inputs(workload, rank=0, scale=1.0, device=None):
    """The seeded numpy columns of a workload at its stated size (times
    `scale`): {"build", "probe"} for the join, {"t"} otherwise.  Both arms of
    the benchmark draw their inputs here, so the reference engine and the GPU
    see the same shapes and, in one process, the same buffers.  `device`
    draws the 200M-row Zipf table on that torch device (a numpy draw of it
    takes about a minute)."""
    from teide_b200 import workloads
    if workload == "join_group":
        b, p = workloads.join_tables(n_probe=int(100_000_000 * scale), seed=3 + 1000 * rank)
        return {"build": b, "probe": p}
    if workload in ("group_radix", "group_sort"):
        return {"t": workloads.zipf_group_table(n=int(200_000_000 * scale), seed=2 + 1000 * rank, device=device)}
    return {"t": workloads.readme_table(n=int(10_000_000 * scale), seed=1 + 1000 * rank)}


def workload_rows(workload, cols):
    """(rows per query, algorithmic bytes per query, bytes the main kernel streams)."""
    if workload == "join_group":
        n = len(cols["probe"]["fk"])
        return n, 16 * len(cols["build"]["pk"]) + 24 * n, 24 * n
    n = len(next(iter(cols["t"].values())))
    return n, 24 * n, 24 * n


def bench_config(workload, rows, alg_bytes, world, scale):
    """The `config` object of a workload's JSON line; both arms print the same one."""
    return {"workload": workload, "rows_per_gpu_per_step": rows, "algorithmic_bytes_per_step": alg_bytes,
            "l2": "inputs larger than L2 (no flush)",
            "parallelism": f"shards{world}" if world > 1 else "single",
            "exchange": ("partial groups merged across ranks (all-gather, or all-to-all by key hash "
                         "when large) inside every step") if world > 1 else None,
            "scale": scale}


def make_tables(td, workload, rank, device, scale=1.0):
    cols = workload_inputs(workload, rank, scale, device)
    tabs = {k: td.table(v) for k, v in cols.items()}
    return (tabs, cols) + workload_rows(workload, cols)


def splay_main(args, td, L, rank, world, local, barrier, max_over_ranks):
    """A splayed table on local disk (the Zipf group-by columns: key, v1, v2 at 50M
    rows, 1.2 GB) read into HBM by td_gpu_splay_load each step: the column
    files come from the page cache into page-locked blocks and are copied to
    the device.  value = column bytes resident per second, whole job."""
    import ctypes as C
    import shutil
    import tempfile
    from teide_b200 import workloads
    L.td_gpu_splay_load.restype = C.c_void_p
    L.td_gpu_splay_load.argtypes = [C.c_char_p]
    n = int(50_000_000 * args.scale)
    c = workloads.zipf_group_table(n=n, seed=2 + 1000 * rank, device="cuda")
    bytes_ = sum(v.nbytes for v in c.values())
    t = td.table(c)
    del c
    root = tempfile.mkdtemp(prefix="td_splay_")
    dirp = os.path.join(root, "t").encode()
    try:
        if L.td_splay_save(t, dirp, None) != 0:
            raise RuntimeError("td_splay_save failed")
        td.release(t)
        for _ in range(args.warmup):
            r = td.check(L.td_gpu_splay_load(dirp), "td_gpu_splay_load")
            L.td_gpu_unpin(r)
            td.release(r)
        barrier()
        clk = Clocks(local).__enter__()
        tc0 = time.monotonic()
        l0 = L.tdg_launch_count()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            r = td.check(L.td_gpu_splay_load(dirp), "td_gpu_splay_load")
            L.td_gpu_unpin(r)
            td.release(r)
        barrier()
        dt = max_over_ranks((time.perf_counter() - t0) / args.steps)
        launches = int(L.tdg_launch_count() - l0)            # the min/max statistics of each column
        tc1 = time.monotonic()
        clk.__exit__(None, None, None)
        value = bytes_ * world / dt / 1e9
        cpu = None
        if rank == 0 and world == 1 and not args.no_cpu_baseline and os.path.exists(REF_LIB):
            from teide_b200.td import Td
            rtd = Td(REF_LIB)
            # the column files, not ".d": its name ids belong to this process's other symbol table
            files = [os.path.join(dirp, f) for f in sorted(os.listdir(dirp)) if not f.startswith(b".")]
            k = 0
            t1 = time.perf_counter()
            while k < 3:
                for f in files:
                    rtd.release(rtd.check(rtd.lib.td_col_load(f), "td_col_load"))
                k += 1
            cdt = (time.perf_counter() - t1) / k
            cpu = {"value": bytes_ / cdt / 1e9, "unit": "GB/s", "cores": os.cpu_count(), "kind": "reference",
                   "sample": f"Teide's td_col_load of the same {len(files)} column files into host memory, "
                             f"mean of {k}"}
    finally:
        shutil.rmtree(root, ignore_errors=True)
    return {
        "metric": METRIC, "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int64/f64", "data": "synthetic",
        "config": {"workload": "splay_load", "rows_per_gpu": n, "bytes_per_gpu": bytes_,
                   "source": "column files in the page cache (written just before)", "scale": args.scale},
        "roofline": None, "roofline_note": "bound by the host read and the host->device link, not by an HBM kernel",
        "e2e": {"value": value, "unit": "GB/s", "h2d_bytes_per_step": bytes_, "d2h_bytes_per_step": 0},
        "gpu_launches": launches, "clocks": clk.summary(tc0, tc1), "cpu_baseline": cpu,
    }


def prepare_query(td, workload, tabs):
    """The workload's DAG, built once (a prepared query); each step executes
    it.  Building a DAG costs microseconds of host calls and no device work."""
    from teide_b200.pipelines import prepared_fused_join_group, prepared_group_sorted, prepared_readme_group
    from teide_b200.td import OP_AVG, OP_COUNT, OP_MAX, OP_MIN, OP_SUM
    aggs5 = [(OP_COUNT, "v1"), (OP_SUM, "v1"), (OP_MIN, "v1"), (OP_MAX, "v1"), (OP_AVG, "v2")]
    if workload == "join_group":
        return prepared_fused_join_group(td, tabs["build"], tabs["probe"], ("qty", "gt", 10), "fk", "pk", ["cat"],
                                         [(OP_SUM, "price"), (OP_COUNT, "price")])
    if workload == "group_radix":
        return prepared_readme_group(td, tabs["t"], ("v1", "gt", 0), ["key"], aggs5)
    if workload == "group_sort":
        return prepared_group_sorted(td, tabs["t"], ("v1", "gt", 0), ["key"], aggs5, "v1_sum", desc=True)
    return prepared_readme_group(td, tabs["t"], ("flag", "eq", 0), ["region"], [(OP_SUM, "amount")])


def run_query(td, workload, tabs, world=1, prepared=None):
    """One step: the prepared query on one GPU.  With several ranks every
    rank runs its shard and the partial groups are merged across ranks
    (teide_b200.shard) inside the step."""
    from teide_b200.td import OP_AVG, OP_COUNT, OP_MAX, OP_MIN, OP_SUM
    if world > 1:
        from teide_b200 import shard
        if workload == "group_sort":
            raise SystemExit("group_sort runs on one GPU (the sharded merge returns unsorted groups)")
        if workload == "join_group":
            return shard.sharded_join_group(td, tabs["build"], tabs["probe"], ("qty", "gt", 10), "fk", "pk",
                                            ["cat"], [(OP_SUM, "price"), (OP_COUNT, "price")])
        if workload == "group_radix":
            return shard.sharded_group(td, tabs["t"], ["key"], [(OP_COUNT, "v1"), (OP_SUM, "v1"), (OP_MIN, "v1"),
                                                               (OP_MAX, "v1"), (OP_AVG, "v2")], pred=("v1", "gt", 0))
        return shard.sharded_group(td, tabs["t"], ["region"], [(OP_SUM, "amount")], pred=("flag", "eq", 0))
    return prepared.run()


def _sub(args, **kw):
    """A copy of the arguments for a sub-measurement (no CPU baseline, no
    end-to-end pass, its own size)."""
    a = argparse.Namespace(**vars(args))
    a.no_cpu_baseline = True
    a.no_e2e = True
    for k, v in kw.items():
        setattr(a, k, v)
    return a


def batch_summary(b):
    p = b.get("plain") or {}
    return {"queries_per_s": b["value"], "plain_queries_per_s": p.get("value"), "speedup": p.get("speedup"),
            "queries": b["config"]["queries_per_step"], "rows_per_step": b["config"]["rows_per_step"],
            "ms_per_step": b["ms_per_step"], "roofline_frac": b["roofline"]["frac"],
            "how": "one persistent kernel replayed as a CUDA graph; plain = one td_execute per query"}


def stats_of(td):
    import ctypes as C

    class St(C.Structure):
        _fields_ = [("h2d", C.c_uint64), ("d2h", C.c_uint64), ("calls", C.c_uint64), ("live", C.c_uint64),
                    ("peak", C.c_uint64), ("gm", C.c_int32), ("jm", C.c_int32), ("fused", C.c_int32),
                    ("pad", C.c_int32)]
    s = St()
    td.lib.td_gpu_last_stats(C.byref(s))
    return s


# ---- batched group-by (4096 independent queries) ---------------------------------------

class Batch:
    """4096 group-by queries (SUM/COUNT/MAX of val by key), one table each:
    rows log-uniform in [1K, 2M], key U[0, K) with K log-uniform in [16, 65536],
    val U[0, 1).  Graphs are built once and executed repeatedly (prepared
    queries); columns are written straight into td vectors."""

    def __init__(self, td, n_queries=4096, seed=4, first=None):
        import ctypes as C
        import numpy as np
        from teide_b200 import workloads
        from teide_b200.td import F64, I64, OP_COUNT, OP_MAX, OP_SUM
        self.td = td
        rows, ks = workloads.batch_shapes(n_queries=n_queries, seed=seed)
        if first:
            rows, ks = rows[:first], ks[:first]
        self.rows = int(rows.sum())
        self.n = len(rows)
        self.tables, self.graphs, self.roots = [], [], []
        for i, (n, k) in enumerate(zip(rows, ks)):
            r = np.random.default_rng(seed * 100_000 + i)
            kv, kview = td.vec_alloc(I64, int(n))
            vv, vview = td.vec_alloc(F64, int(n))
            kview[:] = r.integers(0, int(k), int(n), dtype=np.int64)
            r.random(out=vview)
            t = td.table({"key": kv, "val": vv})
            td.release(kv)
            td.release(vv)
            g = td.graph(t)
            self.roots.append(g.group([g.scan("key")], [OP_SUM, OP_COUNT, OP_MAX], [g.scan("val")] * 3))
            self.tables.append(t)
            self.graphs.append(g)
        self.G = (C.c_void_p * self.n)(*[g.g for g in self.graphs])
        self.R = (C.c_void_p * self.n)(*self.roots)
        if hasattr(td.lib, "td_execute_batch"):       # Teide itself has no batch entry
            td.lib.td_execute_batch.restype = C.c_void_p
            td.lib.td_execute_batch.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]

    def batched(self):
        r = self.td.check(self.td.lib.td_execute_batch(self.G, self.R, self.n), "td_execute_batch")
        self.td.release(r)

    def plain(self):
        """One td_execute per query (one query per launch sequence)."""
        for g, root in zip(self.graphs, self.roots):
            self.td.release(g.execute(root, optimize=False))


def batch_main(args, td, L, rank, world, local, barrier, max_over_ranks):
    import torch
    b = Batch(td, seed=4 + 1000 * rank, first=max(1, int(round(4096 * args.scale))))
    for t in b.tables:
        st = L.td_gpu_pin(t)
        if st:
            raise RuntimeError(f"td_gpu_pin failed: {st}")
    L.tdg_set_timing(0)
    b.batched()                                 # autotune (or load the tuned shape) + graph capture
    clk = Clocks(local).__enter__()
    for _ in range(args.warmup):
        b.batched()
    barrier()
    l0 = L.tdg_launch_count()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    tc0 = time.monotonic()
    ev0.record()
    for _ in range(args.steps):
        b.batched()
    ev1.record()
    torch.cuda.synchronize()
    tc1 = time.monotonic()
    launches = L.tdg_launch_count() - l0
    elapsed = max_over_ranks(ev0.elapsed_time(ev1) / 1e3)
    value = b.n * world * args.steps / elapsed
    # aggregation kernel alone (direct launches with CUDA events, no graph)
    L.tdg_set_timing(1)
    main_ms = []
    for _ in range(max(3, args.steps)):
        b.batched()
        main_ms.append(L.tdg_last_main_ms())
    L.tdg_set_timing(0)
    # plain: the same queries, one td_execute each
    plain = None
    if not args.no_plain:
        b.plain()
        barrier()
        plain_steps = 2
        ev0.record()
        for _ in range(plain_steps):
            b.plain()
        ev1.record()
        torch.cuda.synchronize()
        plain_elapsed = max_over_ranks(ev0.elapsed_time(ev1) / 1e3)
        plain_value = b.n * world * plain_steps / plain_elapsed
        plain = {"value": plain_value, "unit": "queries/s", "steps": plain_steps,
                 "how": "one td_execute per query, same resident tables", "speedup": value / plain_value}
    time.sleep(0.3)
    clk.__exit__(None, None, None)
    # end to end: host tables, every step uploads every query's columns
    e2e = None
    if not args.no_e2e:
        for t in b.tables:
            L.td_gpu_unpin(t)
        L.td_gpu_trim()
        b.batched()
        barrier()
        e2e_steps = args.e2e_steps or 2
        ev0.record()
        for _ in range(e2e_steps):
            b.batched()
        ev1.record()
        torch.cuda.synchronize()
        e2e_elapsed = max_over_ranks(ev0.elapsed_time(ev1) / 1e3)
        s_e2e = stats_of(td)
        e2e = {"value": b.n * world * e2e_steps / e2e_elapsed, "unit": "queries/s",
               "h2d_bytes_per_step": int(s_e2e.h2d), "d2h_bytes_per_step": int(s_e2e.d2h), "steps": e2e_steps}
    hbm, peak_kind = peaks()
    mean_main = statistics.median(main_ms)
    alg = 16 * b.rows
    achieved = alg / (mean_main / 1e3) / 1e9 if mean_main > 0 else None
    line = {
        "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": elapsed / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64/f64", "data": "synthetic",
        "config": {"workload": "batch", "queries_per_step": b.n, "rows_per_step": b.rows,
                   "algorithmic_bytes_per_step": alg, "aggs": "SUM/COUNT/MAX(val) by key",
                   "l2": "inputs larger than L2 (no flush)", "tables": "resident in HBM (td_gpu_pin)",
                   "launch": "td_execute_batch: one persistent kernel, replayed CUDA graph",
                   "parallelism": f"replicas{world}", "scale": args.scale},
        "plain": plain,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": (achieved / hbm) if achieved else None,
                     "traffic": profile_traffic("k_batch_agg_batch.md"), "kernel": "k_batch_agg",
                     "bytes_per_launch": alg, "mean_launch_ms": mean_main, "peak_source": peak_kind},
        "e2e": e2e,
        "gpu_launches": int(launches),
        "clocks": clk.summary(tc0, tc1),
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline and os.path.exists(REF_LIB):
        rtd, q, desc = reference_sample("batch")
        q()
        t0 = time.perf_counter()
        n = 0
        while n < 2 or time.perf_counter() - t0 < 10:
            q()
            n += 1
        dt = (time.perf_counter() - t0) / n
        line["cpu_baseline"] = {"value": BATCH_REF_QUERIES / dt, "unit": "queries/s", "cores": os.cpu_count(),
                                "kind": "reference", "sample": desc + f", mean of {n} runs"}
    return line


BATCH_REF_QUERIES = 512


# ---- served mix (request loop over resident tables) ------------------------------------

def d2h_gbs(nbytes=256 << 20):
    """Device -> page-locked host copy bandwidth of this box (GB/s, best of 3):
    the link every served group-by result crosses."""
    import torch
    src = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    dst = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    best = 0.0
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        dst.copy_(src, non_blocking=True)
        e1.record()
        torch.cuda.synchronize()
        best = max(best, nbytes / (e0.elapsed_time(e1) / 1e3) / 1e9)
    return best


def serve_main(args, td, L, rank, world, local, barrier, max_over_ranks):
    """The served mix over resident tables: 70% filter + group-by on the
    200M-row Zipf table, 30% filter + join + group-by on the 10M / 100M-row
    join tables, each over a random row range of 100K..50M rows, Poisson
    arrivals at 2000 q/s.  The same trace runs through a td_server with
    `slots` slots and with 1 slot (one query at a time): closed loop (all
    submitted at once: throughput at saturation) and open loop (each
    submitted at its arrival time: p50 / p99 latency) at 2000 q/s, and for
    the served form also open loop at 80% of its own closed-loop rate (a load
    it sustains, so the percentiles describe the server rather than a
    growing queue)."""
    import numpy as np
    import torch
    from teide_b200 import serve, workloads
    scale = args.scale
    n_group, n_probe = int(200_000_000 * scale), int(100_000_000 * scale)
    c2 = workloads.zipf_group_table(n=n_group, seed=2 + 1000 * rank, device="cuda")
    b, p = workloads.join_tables(n_probe=n_probe, seed=3 + 1000 * rank, device="cuda")
    tg, tb, tp = td.table(c2), td.table(b), td.table(p)
    del c2, b, p
    torch.cuda.empty_cache()
    for t in (tg, tb, tp):
        st = L.td_gpu_pin(t)
        if st:
            raise RuntimeError(f"td_gpu_pin failed: {st}")
    raw = workloads.serve_requests(args.requests, rate=2000.0, seed=5 + rank, group_rows=n_group,
                                   probe_rows=n_probe,
                                   len_range=(100_000, max(100_000, int(50_000_000 * scale))))
    reqs = [serve.Request(*r) for r in raw]
    serve.build(td, reqs, tg, tb, tp)
    alg = sum(24 * r.n + (16 * 10_000_000 if r.kind == "join" else 0) for r in reqs)
    warm = reqs[:min(len(reqs), 32)]
    out, launches = {}, {}
    clk = Clocks(local).__enter__()
    tc0 = time.monotonic()
    d2h = 0
    for name, slots in (("served", args.slots), ("one_at_a_time", 1)):
        with serve.Server(td, slots=slots) as srv:
            serve.run_closed(srv, warm)                      # warm-up: caches, page-locked result blocks
            barrier()
            s0 = stats_of(td)
            l0 = L.tdg_launch_count()
            closed = serve.run_closed(srv, reqs)
            launches[name] = int(L.tdg_launch_count() - l0)
            lat, makespan, _ = serve.run_open_loop(srv, reqs)
            o = {"closed_qps": len(reqs) / closed, "closed_s": closed,
                 "qps_at_2000": len(reqs) / makespan, "p50_ms_at_2000": float(np.percentile(lat, 50) * 1e3),
                 "p99_ms_at_2000": float(np.percentile(lat, 99) * 1e3), "slots": slots}
            if name == "served":
                rate = 0.8 * o["closed_qps"]
                paced = [serve.Request(r.kind, r.off, r.n, r.threshold, r.arrival * 2000.0 / rate) for r in reqs]
                for r, q in zip(paced, reqs):
                    r.tbl, r.graph, r.root = q.tbl, q.graph, q.root
                lat2, mk2, _ = serve.run_open_loop(srv, paced)
                o["sustained"] = {"offered_qps": rate, "qps": len(reqs) / mk2,
                                  "p50_ms": float(np.percentile(lat2, 50) * 1e3),
                                  "p99_ms": float(np.percentile(lat2, 99) * 1e3)}
            st = srv.stats()
            o["peak_in_flight"] = int(st.peak_in_flight)
            out[name] = o
    tc1 = time.monotonic()
    time.sleep(0.3)
    clk.__exit__(None, None, None)
    # result bytes per request (the group-bys' rows cross the host link)
    for r in reqs[:64]:
        res = td.check(L.td_execute(r.graph.g, r.root), "execute")
        d2h += int(stats_of(td).d2h)
        td.release(res)
    d2h_per_req = d2h / min(len(reqs), 64)
    link = d2h_gbs()
    serve.release(td, reqs)
    for t in (tg, tb, tp):
        L.td_gpu_unpin(t)
        td.release(t)
    sv, one = out["served"], out["one_at_a_time"]
    value = world / max_over_ranks(1.0 / sv["closed_qps"])
    hbm, peak_kind = peaks()
    achieved = alg / sv["closed_s"] / 1e9
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and os.path.exists(REF_LIB):
        _, q, desc = reference_sample("serve")
        secs = q()
        _, threads = reference_engine()
        cpu = {"value": SERVE_REF_REQUESTS / secs, "unit": "queries/s", "cores": threads,
               "kind": "reference", "sample": desc}
    return {
        "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": 1,
        "warmup": len(warm), "ms_per_step": sv["closed_s"] * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64/f64", "data": "synthetic",
        "config": {"workload": "serve", "requests": len(reqs), "arrivals": "Poisson 2000 q/s",
                   "mix": "70% filter+group (200M-row Zipf table), 30% filter+join+group (10M/100M)",
                   "range_rows": "U[100K, 50M]", "tables": "resident in HBM (td_gpu_pin), loaded once",
                   "slots": args.slots, "admission": "FIFO by estimated device bytes vs 90% of free HBM",
                   "algorithmic_bytes": alg, "scale": scale, "timing": "host CLOCK_MONOTONIC per request",
                   "parallelism": f"replicas{world}"},
        "served": sv, "plain": one,
        "speedup_closed_loop": sv["closed_qps"] / one["closed_qps"],
        "result_d2h_bytes_per_request": d2h_per_req, "d2h_link_gbs": link,
        "link_floor_qps": link * 1e9 / d2h_per_req if d2h_per_req else None,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "traffic": None, "kernel": "whole served pipeline (closed loop)", "peak_source": peak_kind},
        "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": int(d2h_per_req * len(reqs)),
                "note": "tables are resident by design; results are host td_t tables"},
        "gpu_launches": launches.get("served"),
        "clocks": clk.summary(tc0, tc1),
        "cpu_baseline": cpu,
    }


def serve_summary(v):
    sv, one = v["served"], v["plain"]
    return {"qps": sv["closed_qps"], "plain_qps": one["closed_qps"], "speedup": v["speedup_closed_loop"],
            "sustained": sv.get("sustained"),
            "at_2000_qps": {"qps": sv["qps_at_2000"], "p50_ms": sv["p50_ms_at_2000"], "p99_ms": sv["p99_ms_at_2000"]},
            "plain_at_2000_qps": {"qps": one["qps_at_2000"], "p50_ms": one["p50_ms_at_2000"],
                                  "p99_ms": one["p99_ms_at_2000"]},
            "requests": v["config"]["requests"], "slots": sv["slots"],
            "result_d2h_bytes_per_request": v["result_d2h_bytes_per_request"], "d2h_link_gbs": v["d2h_link_gbs"],
            "link_floor_qps": v["link_floor_qps"],
            "how": "td_server over resident tables; plain = the same trace through one slot (one query at a time)"}


def serve_small(td, L, n_queries=1024, slots=8, seed=6):
    """The served form on a stream of small group-by requests: the first
    `n_queries` of the batched workload's queries (one table each, rows
    log-uniform in [1K, 2M], 16 to 65536 keys), submitted to td_server at
    once (closed loop: one td_server_submit_many and one td_server_wait_many
    call) against the same requests run one td_execute after another; then
    offered one by one from Python (open loop) at half the served rate, at most
    the one-at-a-time rate, for the latency percentiles.  The server packs same-shape requests that wait behind each
    other into td_execute_batch launches."""
    import numpy as np
    from teide_b200 import serve
    b = Batch(td, seed=seed, first=n_queries)
    for t in b.tables:
        st = L.td_gpu_pin(t)
        if st:
            raise RuntimeError(f"td_gpu_pin failed: {st}")

    class Req:
        __slots__ = ("graph", "root", "arrival", "kind")

    reqs = []
    for g, root in zip(b.graphs, b.roots):
        q = Req()
        q.graph, q.root, q.arrival, q.kind = g, root, 0.0, "group"
        reqs.append(q)
    b.plain()                                           # warm-up: uploads, statistics, plans
    t0 = time.perf_counter()
    b.plain()
    plain_s = time.perf_counter() - t0
    import ctypes as C
    L.td_server_submit_many.restype = C.c_int64
    L.td_server_submit_many.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]
    L.td_server_wait_many.restype = None
    L.td_server_wait_many.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
    tickets = (C.c_int64 * len(reqs))()
    timings = (serve.Timing * len(reqs))()

    def closed_loop(srv):
        # every request submitted and collected with one call each (the results
        # are released inside): the client's per-request cost is not Python's
        t0 = time.monotonic_ns()
        if L.td_server_submit_many(srv.s, b.G, b.R, len(reqs), tickets) != len(reqs):
            raise RuntimeError("td_server_submit_many refused a request")
        L.td_server_wait_many(srv.s, tickets, len(reqs), None, timings)
        if any(t.status for t in timings):
            raise RuntimeError("a served request failed")
        return (max(t.end_ns for t in timings) - t0) / 1e9

    with serve.Server(td, slots=slots) as srv:
        for _ in range(2):
            closed_loop(srv)                            # warm-up: batch plans, host blocks
        closed = min(closed_loop(srv) for _ in range(3))
        # offered one by one from Python: at most the one-at-a-time rate (the
        # load at which plain execution saturates; the Python client's own
        # pacing falls behind from about 20K requests/s)
        rate = min(0.5 * len(reqs) / closed, len(reqs) / plain_s)
        r = np.random.default_rng(seed)
        arrivals = np.cumsum(r.exponential(1.0 / rate, len(reqs)))
        for q, a in zip(reqs, arrivals):
            q.arrival = float(a - arrivals[0])
        lat, makespan, _ = serve.run_open_loop(srv, reqs)
    for t in b.tables:
        L.td_gpu_unpin(t)
    out = {"requests": len(reqs), "slots": slots, "qps": len(reqs) / closed, "plain_qps": len(reqs) / plain_s,
           "speedup": plain_s / closed,
           "sustained": {"offered_qps": rate, "qps": len(reqs) / makespan if makespan else None,
                         "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3)},
           "how": "td_server packs queued same-shape group-by requests into td_execute_batch launches; "
                  "plain = one td_execute per request in arrival order"}
    for g in b.graphs:
        g.free()
    for t in b.tables:
        td.release(t)
    return out


# ---- CPU reference ---------------------------------------------------------------------

SERVE_REF_ROWS, SERVE_REF_REQUESTS = 60_000_000, 16


def serve_reference(td):
    """Teide one query at a time over a sample of the served mix: 16 requests
    drawn like the GPU trace (ranges U[100K, 50M]) from 60M-row tables of the
    same shapes.  Each range is copied into its own table before the clock
    starts; the query runs Teide's filter -> group and filter -> join -> group
    graphs.  The returned callable gives the seconds spent in queries."""
    from teide_b200.pipelines import const
    from teide_b200 import serve as sv
    from teide_b200 import workloads
    c2 = workloads.zipf_group_table(n=SERVE_REF_ROWS, seed=32)
    b, p = workloads.join_tables(n_build=10_000_000, n_probe=SERVE_REF_ROWS, seed=33)
    raw = workloads.serve_requests(SERVE_REF_REQUESTS, seed=55, group_rows=SERVE_REF_ROWS,
                                     probe_rows=SERVE_REF_ROWS)
    bt = td.table(b)

    def run(graph_tbl, build):
        g = td.graph(graph_tbl)
        try:
            return g.execute(build(g))
        finally:
            g.free()

    def q():
        total = 0.0
        for kind, off, n, thr, _ in raw:
            src = c2 if kind == "group" else p
            tt = td.table({k: v[off:off + n] for k, v in src.items()})
            t0 = time.perf_counter()
            col = "v1" if kind == "group" else "qty"
            ft = run(tt, lambda g: g.filter(g.const_table(tt), g.op("gt", g.scan(col), const(g, thr))))
            if kind == "group":
                r = run(ft, lambda g: g.group([g.scan("key")], [a for a, _ in sv.GROUP_AGGS],
                                              [g.scan(x) for _, x in sv.GROUP_AGGS]))
            else:
                jt = run(ft, lambda g: g.join(g.const_table(ft), [g.scan("fk")], g.const_table(bt),
                                              [g.scan("pk")], 0))
                r = run(jt, lambda g: g.group([g.scan("cat")], [a for a, _ in sv.JOIN_AGGS],
                                              [g.scan(x) for _, x in sv.JOIN_AGGS]))
                td.release(jt)
            td.release(r)
            td.release(ft)
            total += time.perf_counter() - t0
            td.release(tt)
        return total
    desc = (f"{SERVE_REF_REQUESTS} requests of the served mix over 60M-row tables of the same shapes, "
            "one at a time (filter graph then group / join + group graphs)")
    return td, q, desc


REF_BUILD = ("gcc -std=c17 -O3 -march=x86-64-v3 -DNDEBUG: the reference's release flags, with "
             "x86-64-v3 (AVX2) in place of -march=native so one binary runs on every host")


@functools.lru_cache(maxsize=1)
def reference_engine():
    """Teide's own engine (compiled from its sources into oracle/_ref) and the
    number of threads its td_execute runs on (the pool's workers + caller)."""
    import ctypes as C
    from teide_b200.td import Td
    td = Td(REF_LIB)
    td.lib.td_thread_count.restype = C.c_uint32
    return td, int(td.lib.td_thread_count())


def reference_sample(workload, cols=None, scale=1.0):
    """Teide's CPU engine on one query of the workload at the same size as
    the GPU arm: returns (td, query callable, description).  `cols` are the
    GPU arm's own input arrays when this runs in its process; otherwise they
    are drawn from the same generators."""
    from teide_b200.pipelines import join_then_group, two_graph_group, two_graph_group_sorted
    from teide_b200.td import OP_AVG, OP_COUNT, OP_MAX, OP_MIN, OP_SUM
    td, threads = reference_engine()
    if workload == "serve":
        return serve_reference(td)
    if workload == "batch":
        b = Batch(td, first=BATCH_REF_QUERIES)
        desc = (f"the first {b.n} of the 4096 queries ({b.rows / 1e6:.1f}M rows), one td_execute each")
        return td, b.plain, desc
    if cols is None:
        cols = workload_inputs(workload, 0, scale, device="cpu")
    if workload == "join_group":
        bt, pt = td.table(cols["build"]), td.table(cols["probe"])

        def q():
            join_then_group(td, bt, pt, ("qty", "gt", 10), "fk", "pk", ["cat"],
                            [(OP_SUM, "price"), (OP_COUNT, "price")], as_dict=False)
        desc = (f"build {len(cols['build']['pk']) / 1e6:g}M + probe {len(cols['probe']['fk']) / 1e6:g}M rows per "
                "query: Teide's filter + join graph, then the group graph over the joined table")
    else:
        t = td.table(cols["t"])
        n = len(next(iter(cols["t"].values())))
        aggs5 = [(OP_COUNT, "v1"), (OP_SUM, "v1"), (OP_MIN, "v1"), (OP_MAX, "v1"), (OP_AVG, "v2")]
        if workload == "group_radix":
            def q():
                two_graph_group(td, t, ("v1", "gt", 0), ["key"], aggs5, as_dict=False)
            desc = f"{n / 1e6:g}M rows per query: Teide's filter graph, then the group graph"
        elif workload == "group_sort":
            def q():
                two_graph_group_sorted(td, t, ("v1", "gt", 0), ["key"], aggs5, "v1_sum", desc=True)
            desc = f"{n / 1e6:g}M rows per query, group result sorted by v1_sum DESC"
        else:
            def q():
                two_graph_group(td, t, ("flag", "eq", 0), ["region"], [(OP_SUM, "amount")], as_dict=False)
            desc = f"{n / 1e6:g}M rows per query: Teide's filter graph, then the group graph"
    return td, q, desc + f"; {threads} threads; {REF_BUILD}"


def reference_splay(args):
    """Teide's td_splay_load of a 50M-row splayed table (the Zipf group-by columns) into host memory."""
    import ctypes as C
    import shutil
    import tempfile
    from teide_b200 import workloads
    from teide_b200.td import Td
    td = Td(REF_LIB)
    td.lib.td_splay_load.restype = C.c_void_p
    n = int(50_000_000 * args.scale)
    c = workloads.zipf_group_table(n=n, seed=2)
    bytes_ = sum(v.nbytes for v in c.values())
    t = td.table(c)
    del c
    root = tempfile.mkdtemp(prefix="td_splay_ref_")
    dirp = os.path.join(root, "t").encode()
    try:
        if td.lib.td_splay_save(t, dirp, None) != 0:
            raise RuntimeError("td_splay_save failed")
        td.release(t)
        for _ in range(args.warmup):
            td.release(td.check(td.lib.td_splay_load(dirp), "td_splay_load"))
        t0 = time.perf_counter()
        for _ in range(args.steps):
            td.release(td.check(td.lib.td_splay_load(dirp), "td_splay_load"))
        dt = (time.perf_counter() - t0) / args.steps
    finally:
        shutil.rmtree(root, ignore_errors=True)
    v = bytes_ / dt / 1e9
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "GB/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "int64/f64", "data": "synthetic",
        "config": {"workload": "splay_load", "rows_per_gpu": n, "bytes_per_gpu": bytes_, "scale": args.scale},
        "cpu_baseline": {"value": v, "unit": "GB/s", "cores": os.cpu_count(), "kind": "reference",
                         "sample": "the whole table, td_splay_load into host memory"},
        "e2e": {"value": v, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def reference_arm(args):
    """Teide's own CPU engine on the same workload, sizes and config as the
    GPU arm (rank 0 only; other ranks exit without work)."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    if not os.path.exists(REF_LIB):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libteide_ref.so not built"}))
        return
    if args.workload == "splay_load":
        return reference_splay(args)
    td, q, desc = reference_sample(args.workload, scale=args.scale)
    if args.workload == "serve":                 # q() reports its own query seconds
        for _ in range(min(args.warmup, 1)):
            q()
        dt = sum(q() for _ in range(max(1, min(args.steps, 2)))) / max(1, min(args.steps, 2))
        rows, config = SERVE_REF_REQUESTS, {"workload": "serve", "sample": desc}
    elif args.workload == "batch":
        for _ in range(args.warmup):
            q()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            q()
        dt = (time.perf_counter() - t0) / args.steps
        rows, config = BATCH_REF_QUERIES, {"workload": "batch", "sample": desc}
    else:
        for _ in range(args.warmup):
            q()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            q()
        dt = (time.perf_counter() - t0) / args.steps
        rows, alg, _ = workload_rows(args.workload, workload_inputs_shape(args.workload, args.scale))
        config = bench_config(args.workload, rows, alg, args.gpus, args.scale)
    v = rows / dt
    unit = "queries/s" if args.workload in ("batch", "serve") else "rows/s"
    _, threads = reference_engine()
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": unit, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64/f64", "data": "synthetic",
        "config": config, "tables": "host memory (Teide's heap)",
        "cpu_baseline": {"value": v, "unit": unit, "cores": threads, "kind": "reference",
                         "sample": f"the whole workload, every step; {desc}"},
        "e2e": {"value": v, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def workload_inputs_shape(workload, scale=1.0):
    """Row counts of a workload's inputs, without drawing them."""
    import numpy as np
    if workload == "join_group":
        return {"build": {"pk": np.empty(10_000_000)}, "probe": {"fk": np.empty(int(100_000_000 * scale))}}
    n = int((200_000_000 if workload in ("group_radix", "group_sort") else 10_000_000) * scale)
    return {"t": {"key": np.empty(n, dtype=np.uint8)}}


# ---- GPU arm -------------------------------------------------------------------------------

def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="teide_b200", choices=["teide_b200", "reference"])
    ap.add_argument("--workload", default="join_group", choices=["join_group", "group_radix", "group_sort", "readme_group", "batch",
                                                        "serve", "splay_load"])
    ap.add_argument("--e2e-steps", type=int, default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-table (upload) pass")
    ap.add_argument("--no-plain", action="store_true", help="batch: skip the one-query-per-launch pass")
    ap.add_argument("--requests", type=int, default=2000, help="serve: requests in the trace")
    ap.add_argument("--slots", type=int, default=8, help="serve: queries in flight at once")
    ap.add_argument("--scale", type=float, default=1.0,
                    help="fraction of the workload size (smaller cases for profiler captures)")
    ap.add_argument("--no-extra", action="store_true",
                    help="join_group: skip the batch and serve measurements added to the line")
    ap.add_argument("--batch-scale", type=float, default=0.25,
                    help="join_group line: fraction of the 4096 batched queries measured")
    ap.add_argument("--serve-requests", type=int, default=400,
                    help="join_group line: requests in the served-mix trace")
    args = ap.parse_args()
    if args.impl == "reference":
        return reference_arm(args)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    os.environ["TD_GPU_DEVICE"] = str(local)
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    import teide_b200
    td = teide_b200.load()
    L = td.lib
    L.tdg_set_timing.argtypes = [__import__("ctypes").c_int32]
    L.tdg_last_main_ms.restype = __import__("ctypes").c_float
    L.tdg_last_build_ms.restype = __import__("ctypes").c_float
    L.tdg_last_sort_ms.restype = __import__("ctypes").c_float
    L.tdg_launch_count.restype = __import__("ctypes").c_uint64
    L.td_gpu_pin.argtypes = [__import__("ctypes").c_void_p]
    L.td_gpu_unpin.argtypes = [__import__("ctypes").c_void_p]
    L.tdg_set_timing(1)

    def barrier():
        if dist:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if not dist:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    if args.workload in ("batch", "serve", "splay_load"):
        fn = {"batch": batch_main, "serve": serve_main, "splay_load": splay_main}[args.workload]
        line = fn(args, td, L, rank, world, local, barrier, max_over_ranks)
        if rank == 0:
            print(json.dumps(line))
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    tabs, cols, rows, alg_bytes, main_bytes = make_tables(td, args.workload, rank, "cuda", args.scale)
    torch.cuda.empty_cache()

    # ---- resident: tables pinned in HBM ----
    for t in tabs.values():
        st = L.td_gpu_pin(t)
        if st:
            raise RuntimeError(f"td_gpu_pin failed: {st}")
    prep = prepare_query(td, args.workload, tabs) if world == 1 else None
    clk = Clocks(local).__enter__()
    for _ in range(args.warmup):
        run_query(td, args.workload, tabs, world, prep)
    barrier()
    l0 = L.tdg_launch_count()
    main_ms, build_ms, sort_ms = [], [], []
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    tc0 = time.monotonic()
    ev0.record()
    for _ in range(args.steps):
        run_query(td, args.workload, tabs, world, prep)
        main_ms.append(L.tdg_last_main_ms())
        build_ms.append(L.tdg_last_build_ms())
        sort_ms.append(L.tdg_last_sort_ms())
    ev1.record()
    torch.cuda.synchronize()
    tc1 = time.monotonic()
    time.sleep(0.3)
    clk.__exit__(None, None, None)
    elapsed = ev0.elapsed_time(ev1) / 1e3
    launches = L.tdg_launch_count() - l0
    s_res = stats_of(td)
    barrier()
    elapsed = max_over_ranks(elapsed)
    value = rows * world * args.steps / elapsed

    # ---- end to end: host tables, uploads inside every step ----
    e2e = None
    if not args.no_e2e:
        for t in tabs.values():
            L.td_gpu_unpin(t)
        L.td_gpu_trim()
        e2e_steps = args.e2e_steps or args.steps
        run_query(td, args.workload, tabs, world, prep)    # page-locks the host columns once
        barrier()
        ev0.record()
        for _ in range(e2e_steps):
            run_query(td, args.workload, tabs, world, prep)
        ev1.record()
        torch.cuda.synchronize()
        e2e_elapsed = max_over_ranks(ev0.elapsed_time(ev1) / 1e3)
        s_e2e = stats_of(td)
        e2e = {"value": rows * world * e2e_steps / e2e_elapsed, "unit": "rows/s",
               "h2d_bytes_per_step": int(s_e2e.h2d), "d2h_bytes_per_step": int(s_e2e.d2h), "steps": e2e_steps}

    hbm, peak_kind = peaks()
    mean_main = sum(main_ms) / len(main_ms) if main_ms else 0.0
    achieved = main_bytes / (mean_main / 1e3) / 1e9 if mean_main > 0 else None
    prof = {"join_group": "k_probe_vec_join_group.md", "group_radix": "k_group_vec_part_agg_group_radix.md",
            "group_sort": "k_group_vec_part_agg_group_radix.md",
            "readme_group": "k_group_vec_readme_group.md"}[args.workload]
    line = {
        "metric": METRIC, "value": value, "unit": "rows/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": elapsed / args.steps * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int64/f64", "data": "synthetic",
        "config": bench_config(args.workload, rows, alg_bytes, world, args.scale),
        "tables": "resident in HBM (td_gpu_pin)",
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": (achieved / hbm) if achieved else None, "traffic": profile_traffic(prof),
                     "kernel": {"join_group": "k_probe_vec (fused probe + aggregate)",
                                "group_radix": "k_group_vec + k_part_agg (hot slots in shared memory, cold rows "
                                               "partitioned by slot range and aggregated per partition)",
                                "group_sort": "k_group_vec + k_part_agg (the group-by; the sort is sort_ms)",
                                "readme_group": "k_group_vec (one key, 16-byte column loads)"}[args.workload],
                     "bytes_per_launch": main_bytes,
                     "mean_launch_ms": mean_main, "peak_source": peak_kind,
                     "step_frac": alg_bytes / (elapsed / args.steps) / 1e9 / hbm,
                     "build_ms": (sum(build_ms) / len(build_ms)) if build_ms and build_ms[0] else None},
        "e2e": e2e,
        "gpu_launches": int(launches),
        "clocks": clk.summary(tc0, tc1),
        "resident_h2d_bytes_per_step": int(s_res.h2d),
    }
    if args.workload == "group_sort" and sort_ms:
        line["sort_ms"] = sum(sort_ms) / len(sort_ms)      # tdg_sort_perm: the 5.9M-row permutation
    if rank == 0 and world == 1 and not args.no_cpu_baseline and os.path.exists(REF_LIB):
        # Teide's engine on the same input arrays and the same query as every
        # GPU step: one warm-up, then whole queries until about 10 s have passed.
        rtd, q, desc = reference_sample(args.workload, cols)
        q()
        t0 = time.perf_counter()
        n = 0
        while n < 2 or time.perf_counter() - t0 < 10:
            q()
            n += 1
        dt = (time.perf_counter() - t0) / n
        _, threads = reference_engine()
        line["cpu_baseline"] = {"value": rows / dt, "unit": "rows/s", "cores": threads,
                                "kind": "reference", "sample": f"the whole workload, mean of {n} queries; {desc}"}
    if prep:
        prep.free()
    for t in tabs.values():
        L.td_gpu_unpin(t)
        td.release(t)
    del tabs, cols
    L.td_gpu_trim()
    # the metric's second half, measured in the same run: the batched form
    # (config 4) and the served form (config 5), each against one query at a time
    if world == 1 and args.workload == "join_group" and not args.no_extra:
        line["batch"] = batch_summary(batch_main(_sub(args, scale=args.batch_scale), td, L, rank, world, local,
                                                 barrier, max_over_ranks))
        L.td_gpu_trim()
        small = serve_small(td, L)
        L.td_gpu_trim()
        line["serve"] = serve_summary(serve_main(_sub(args, requests=args.serve_requests), td, L, rank, world,
                                                 local, barrier, max_over_ranks))
        line["serve"]["small_requests"] = small
    if rank == 0:
        print(json.dumps(line))
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
