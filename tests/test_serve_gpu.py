"""The request loop on the GPU: every result is the same alone and in the mix.

A scaled-down served mix (group table 3M rows of the Zipf-key shape, build
200K / probe 3M rows of the join shape, ranges of 10K..1M rows, random
thresholds) runs once query by query on the calling thread, then all at once
through a server with 8 slots.  Every result is checked against the oracle:
integer columns exactly, F64 columns within 1e-12 * max(|want|, sum |x|) per
group (their summation order depends on atomics); alone and in the mix, the
integer columns are also identical to each other."""
import numpy as np
import pytest

import oracle
from teide_b200 import serve, workloads
from teide_b200.pipelines import f64_tolerance_ok
from teide_b200.td import OP_AVG, OP_COUNT, OP_MAX, OP_MIN, OP_SUM

pytestmark = pytest.mark.gpu

N_GROUP, N_BUILD, N_PROBE = 3_000_000, 200_000, 3_000_000


@pytest.fixture(scope="module")
def tables(gpu):
    c2 = workloads.zipf_group_table(n=N_GROUP, seed=52)
    b, p = workloads.join_tables(n_build=N_BUILD, n_probe=N_PROBE, seed=53)
    tg, tb, tp = gpu.table(c2), gpu.table(b), gpu.table(p)
    gpu.lib.td_gpu_pin.argtypes = [serve.P]
    gpu.lib.td_gpu_unpin.argtypes = [serve.P]
    for t in (tg, tb, tp):
        assert gpu.lib.td_gpu_pin(t) == 0
    yield gpu, (c2, b, p), (tg, tb, tp)
    for t in (tg, tb, tp):
        gpu.lib.td_gpu_unpin(t)
        gpu.release(t)


def _requests(n, seed):
    raw = workloads.serve_requests(n, rate=1e9, seed=seed, group_rows=N_GROUP, probe_rows=N_PROBE,
                                     len_range=(10_000, 1_000_000))
    return [serve.Request(*r) for r in raw]


def _canon(d, kind):
    return oracle.canonical(d, by=["key"] if kind == "group" else ["cat"])


def _want(c2, b, p, r):
    """The oracle's result of request r (canonical order) and, per F64
    column, the scale of the tolerance rule (sum |x| for SUM, / count for AVG)."""
    sl = slice(r.off, r.off + r.n)
    if r.kind == "group":
        m = c2["v1"][sl] > r.threshold
        keys = {"key": c2["key"][sl]}
        aggs = [(OP_COUNT, "v1", None), (OP_SUM, "v1", c2["v1"][sl]), (OP_MIN, "v1", c2["v1"][sl]),
                (OP_MAX, "v1", c2["v1"][sl]), (OP_AVG, "v2", c2["v2"][sl])]
    else:
        left = {k: v[sl] for k, v in p.items()}
        j = oracle.join(left, b, ["fk"], ["pk"], 0, lmask=left["qty"] > r.threshold)
        m = None
        keys = {"cat": j["cat"]}
        aggs = [(OP_SUM, "price", j["price"]), (OP_COUNT, "price", None)]
    return _canon(oracle.group(keys, aggs, m), r.kind), oracle.abs_bounds(keys, aggs, m)


def _same(got, want, bounds, what):
    """Integers exact; F64 within 1e-12 * max(|want|, bound) per group."""
    assert list(got) == list(want), what
    for k in want:
        if k in bounds:
            assert f64_tolerance_ok(got[k], want[k], bounds[k]), (what, k)
        else:
            assert np.array_equal(got[k], want[k]), (what, k)


def test_alone_equals_mix(tables):
    """Each of 48 requests run alone (the calling thread, no shared build)
    and in the mix (8 slots; the join requests share one kept payload map)
    matches the oracle, and the two results agree exactly on integers."""
    td, (c2, b, p), (tg, tb, tp) = tables
    reqs = _requests(48, seed=7)
    serve.build(td, reqs, tg, tb, tp)
    try:
        alone = []
        for r in reqs:
            res = td.check(td.lib.td_execute(r.graph.g, r.root), "alone")
            alone.append(_canon(td.table_dict(res), r.kind))
            td.release(res)
        with serve.Server(td, slots=8) as s:
            ts = [s.submit(r.graph, r.root) for r in reqs]
            for i, (r, t) in enumerate(zip(reqs, ts)):
                res, tm = s.wait(t)
                assert tm.status == 0, (i, tm.status)
                mix = _canon(td.table_dict(res), r.kind)
                td.release(res)
                want, bounds = _want(c2, b, p, r)
                what = f"request {i} ({r.kind} [{r.off}, +{r.n}) t={r.threshold})"
                _same(alone[i], want, bounds, what + " alone")
                _same(mix, want, bounds, what + " in the mix")
                for k in want:
                    if k not in bounds:
                        assert np.array_equal(alone[i][k], mix[k]), (what, k)
            st = s.stats()
            assert st.completed == len(reqs) and st.peak_in_flight >= 2
    finally:
        serve.release(td, reqs)


def test_mix_matches_oracle(tables):
    td, (c2, b, p), (tg, tb, tp) = tables
    reqs = _requests(12, seed=11)
    serve.build(td, reqs, tg, tb, tp)
    try:
        with serve.Server(td, slots=4) as s:
            ts = [s.submit(r.graph, r.root) for r in reqs]
            for r, t in zip(reqs, ts):
                res, tm = s.wait(t)
                assert tm.status == 0
                got = _canon(td.table_dict(res), r.kind)
                td.release(res)
                want, bounds = _want(c2, b, p, r)
                _same(got, want, bounds, f"{r.kind} [{r.off}, +{r.n}) t={r.threshold}")
    finally:
        serve.release(td, reqs)


def test_shared_build_follows_the_build_table(gpu):
    """Served join queries keep one payload map per resident build side; a
    new build table -- after the old one is unpinned and freed, so its
    device memory may be handed out again -- must get its own map, never the
    old one: results follow the new table's values."""
    b, p = workloads.join_tables(n_build=200_000, n_probe=1_000_000, seed=61)
    pt = gpu.table(p)
    gpu.lib.td_gpu_pin.argtypes = [serve.P]
    gpu.lib.td_gpu_unpin.argtypes = [serve.P]
    assert gpu.lib.td_gpu_pin(pt) == 0
    try:
        for trial in range(3):
            bb = dict(b)
            bb["cat"] = (b["cat"] * (trial + 1) + trial) % 1000       # same keys, other group slots
            bt = gpu.table(bb)
            assert gpu.lib.td_gpu_pin(bt) == 0
            reqs = [serve.Request("join", 0, len(p["fk"]), t, 0.0) for t in (5, 40, 90)]
            serve.build(gpu, reqs, None, bt, pt)
            with serve.Server(gpu, slots=2) as s:
                ts = [s.submit(r.graph, r.root) for r in reqs]
                for r, t in zip(reqs, ts):
                    res, tm = s.wait(t)
                    assert tm.status == 0
                    got = _canon(gpu.table_dict(res), "join")
                    gpu.release(res)
                    want, bounds = _want(None, bb, p, r)
                    _same(got, want, bounds, f"trial {trial} t={r.threshold}")
            serve.release(gpu, reqs)
            gpu.lib.td_gpu_unpin(bt)
            gpu.release(bt)
    finally:
        gpu.lib.td_gpu_unpin(pt)
        gpu.release(pt)


def test_budget_serializes_and_stays_correct(tables):
    td, (c2, b, p), (tg, tb, tp) = tables
    reqs = _requests(10, seed=13)
    serve.build(td, reqs, tg, tb, tp)
    try:
        for slots, budget in ((8, 1), (8, 0)):
            with serve.Server(td, slots=slots, hbm_budget=budget) as s:
                ts = [s.submit(r.graph, r.root) for r in reqs]
                for i, (r, t) in enumerate(zip(reqs, ts)):
                    p_, tm = s.wait(t)
                    assert tm.status == 0
                    got = _canon(td.table_dict(p_), r.kind)
                    td.release(p_)
                    want, bounds = _want(c2, b, p, r)
                    _same(got, want, bounds, f"request {i} budget {budget}")
                if budget == 1:
                    assert s.stats().peak_in_flight == 1
    finally:
        serve.release(td, reqs)


def test_small_group_requests_are_batched(gpu):
    """Small group-by requests of one shape (one integer key, SUM/COUNT/MAX
    of one value column, over tables of different sizes) queued behind each
    other run as td_execute_batch launches: several requests share one start
    time, and every request's table has the columns and rows td_execute
    gives alone (keys, counts and MAX exactly, SUM within the 1e-12 rule).
    A request of another shape in the middle ends the batch before it and
    runs alone."""
    from teide_b200.td import OP_COUNT as CNT, OP_MAX as MX, OP_SUM as SM
    r = np.random.default_rng(71)
    datas = []
    for i in range(96):
        n = int(r.integers(1_000, 300_000))
        k = int(r.integers(4, 40_000))
        key = r.integers(0, k, n, dtype=np.int64)
        datas.append({"key": key, "val": r.random(n) * 50.0})
    tabs = [gpu.table(d) for d in datas]
    gpu.lib.td_gpu_pin.argtypes = [serve.P]
    gpu.lib.td_gpu_unpin.argtypes = [serve.P]
    for t in tabs:
        assert gpu.lib.td_gpu_pin(t) == 0
    graphs, roots = [], []
    for i, t in enumerate(tabs):
        g = gpu.graph(t)
        if i == 40:                                   # another shape: MIN as well, two value columns
            roots.append(g.group([g.scan("key")], [SM, MX], [g.scan("val"), g.scan("key")]))
        else:
            roots.append(g.group([g.scan("key")], [SM, CNT, MX], [g.scan("val")] * 3))
        graphs.append(g)
    try:
        alone = []
        for g, root in zip(graphs, roots):
            res = g.execute(root)
            alone.append(gpu.table_dict(res))
            gpu.release(res)
        with serve.Server(gpu, slots=1) as srv:
            # the first request occupies the single slot; the rest queue behind it
            tickets = [srv.submit(g, root) for g, root in zip(graphs, roots)]
            got, starts = [], []
            for t in tickets:
                res, tm = srv.wait(t)
                assert tm.status == 0
                got.append(gpu.table_dict(res))
                starts.append(tm.start_ns)
                gpu.release(res)
        assert len(set(starts)) < len(starts) // 4, "requests were not batched"
        for i, (a, b) in enumerate(zip(alone, got)):
            assert list(a) == list(b), i
            for name in a:
                if a[name].dtype.kind == "f" and name.endswith("_sum"):
                    absum = oracle.group({"key": datas[i]["key"]}, [(SM, "val", np.abs(datas[i]["val"]))])["val_sum"]
                    assert f64_tolerance_ok(b[name], a[name], absum), (i, name)
                else:
                    assert np.array_equal(a[name], b[name]), (i, name)
    finally:
        for g in graphs:
            g.free()
        for t in tabs:
            gpu.lib.td_gpu_unpin(t)
            gpu.release(t)


def test_submit_many_and_wait_many(gpu):
    """td_server_submit_many / td_server_wait_many: one call for n requests
    each way; every result equals td_execute alone."""
    import ctypes as C
    from teide_b200.td import OP_COUNT as CNT, OP_SUM as SM
    L = gpu.lib
    L.td_server_submit_many.restype = C.c_int64
    L.td_server_submit_many.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]
    L.td_server_wait_many.restype = None
    L.td_server_wait_many.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p]
    r = np.random.default_rng(72)
    datas = [{"key": r.integers(0, 500, 20_000, dtype=np.int64), "val": r.integers(-9, 9, 20_000, dtype=np.int64)}
             for _ in range(24)]
    tabs = [gpu.table(d) for d in datas]
    graphs = [gpu.graph(t) for t in tabs]
    roots = [g.group([g.scan("key")], [SM, CNT], [g.scan("val")] * 2) for g in graphs]
    try:
        n = len(graphs)
        G = (C.c_void_p * n)(*[g.g for g in graphs])
        R = (C.c_void_p * n)(*roots)
        tickets = (C.c_int64 * n)()
        results = (C.c_void_p * n)()
        timings = (serve.Timing * n)()
        with serve.Server(gpu, slots=4) as srv:
            assert L.td_server_submit_many(srv.s, G, R, n, tickets) == n
            L.td_server_wait_many(srv.s, tickets, n, results, timings)
        for i in range(n):
            assert timings[i].status == 0
            got = gpu.table_dict(results[i])
            gpu.release(results[i])
            want = oracle.group({"key": datas[i]["key"]}, [(SM, "val", datas[i]["val"]), (CNT, "val", None)])
            for k in want:
                assert np.array_equal(got[k], want[k]), (i, k)
    finally:
        for g in graphs:
            g.free()
        for t in tabs:
            gpu.release(t)
