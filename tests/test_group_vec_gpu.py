"""The plain group-by's vector form (one 8-byte key, every column read with
16-byte loads; shared-memory accumulators or the global record array) and
its fallbacks: odd row counts (the last pair is half full), negative key
ranges, a table view starting at an odd row (columns not 16-byte aligned:
the general kernel runs), no filter, one and two filter terms, COUNT only
and F64 / I64 SUM, MIN and MAX -- each against the oracle."""
import numpy as np
import pytest

import oracle
from teide_b200.pipelines import const, f64_tolerance_ok
from teide_b200 import serve
from teide_b200.td import OP_AVG, OP_COUNT, OP_MAX, OP_MIN, OP_SUM

pytestmark = pytest.mark.gpu


def _data(n, seed, lo=0, span=64):
    r = np.random.default_rng(seed)
    return {"flag": r.integers(0, 4, n, dtype=np.int64),
            "region": r.integers(lo, lo + span, n, dtype=np.int64),
            "amount": r.random(n) * 1000.0,
            "qty": r.integers(-500, 500, n, dtype=np.int64)}


def _run(td, tbl, preds, aggs):
    g = td.graph(tbl)
    try:
        p = None
        for c, op, k in preds:
            q = g.op(op, g.scan(c), const(g, k))
            p = q if p is None else g.op("and", p, q)
        f = (lambda v: v) if p is None else (lambda v: g.filter(v, p))
        r = g.execute(g.group([f(g.scan("region"))], [a for a, _ in aggs], [f(g.scan(n)) for _, n in aggs]),
                      optimize=True)
    finally:
        g.free()
    out = td.table_dict(r)
    td.release(r)
    return out


def _want(d, preds, aggs):
    m = np.ones(len(d["region"]), bool)
    for c, op, k in preds:
        m &= oracle.compare(op, d[c], k)
    keys = {"region": d["region"][m]}
    a = [(op, n, None if op == OP_COUNT else d[n][m]) for op, n in aggs]
    want = oracle.group(keys, a)
    want["_abs"] = oracle.abs_bounds(keys, a)
    return want


def _same(got, want):
    """Integers and F64 MIN/MAX exact; F64 SUM/AVG by the 1e-12 rule, with
    the bounds _want put under "_abs"."""
    bounds = want.pop("_abs", {})
    assert list(got) == list(want)
    for k in want:
        if k in bounds:
            assert f64_tolerance_ok(got[k], want[k], bounds[k]), k
        else:
            assert np.array_equal(got[k], want[k]), k


CASES = [
    ([("flag", "eq", 0)], [(OP_SUM, "amount")]),
    ([], [(OP_COUNT, "amount")]),
    ([], [(OP_SUM, "amount"), (OP_MAX, "amount"), (OP_MIN, "amount")]),
    ([("flag", "eq", 1), ("qty", "lt", 100)], [(OP_COUNT, "qty")]),
    ([("qty", "ge", -20), ("qty", "le", 300)], [(OP_SUM, "qty"), (OP_MIN, "qty"), (OP_MAX, "qty")]),
    ([("amount", "gt", 250.0)], [(OP_SUM, "qty"), (OP_COUNT, "qty"), (OP_AVG, "qty")]),
    ([("flag", "ne", 2)], [(OP_SUM, "amount"), (OP_AVG, "amount"), (OP_COUNT, "amount")]),
]


@pytest.mark.parametrize("preds,aggs", CASES)
@pytest.mark.parametrize("n,lo,span", [(400_001, 0, 64), (400_000, -37, 64), (3, 5, 64),
                                       (400_001, -50_000, 150_000)])
def test_vector_group_shapes(gpu, preds, aggs, n, lo, span):
    """span 64: shared-memory accumulators; span 150000: the global record
    array (a direct array too large for shared memory, too few rows to sample
    hot slots)."""
    d = _data(n, seed=91 + n % 7, lo=lo, span=span)
    t = gpu.table(d)
    try:
        _same(_run(gpu, t, preds, aggs), _want(d, preds, aggs))
    finally:
        gpu.release(t)


def test_unaligned_view_falls_back(gpu):
    d = _data(300_000, seed=92)
    t = gpu.table(d)
    view = serve.table_slice(gpu, t, 1, 250_001)          # starts 8 bytes into each column
    try:
        preds, aggs = CASES[0]
        sub = {k: v[1:250_002] for k, v in d.items()}
        _same(_run(gpu, view, preds, aggs), _want(sub, preds, aggs))
    finally:
        gpu.release(view)
        gpu.release(t)


def test_wide_key_range_takes_other_kernels(gpu):
    """A key range too wide for shared memory takes the global-array or hash
    kernel (hash groups come back in slot order, so rows compare sorted)."""
    d = _data(500_000, seed=93, lo=-1_000_000, span=2_000_000)
    t = gpu.table(d)
    try:
        preds, aggs = CASES[0]
        want = _want(d, preds, aggs)          # already in ascending key order, like its bounds
        _same(oracle.canonical(_run(gpu, t, preds, aggs), by=["region"]), want)
    finally:
        gpu.release(t)


AGGS5 = [(OP_COUNT, "qty"), (OP_SUM, "qty"), (OP_MIN, "qty"), (OP_MAX, "qty"), (OP_AVG, "amount")]


@pytest.mark.parametrize("preds,aggs", [
    ([("flag", "ne", 3)], AGGS5),
    ([], [(OP_COUNT, "qty")]),
    ([("qty", "gt", 0)], [(OP_SUM, "amount"), (OP_MIN, "amount"), (OP_MAX, "amount")]),
])
@pytest.mark.parametrize("n,lo,span", [(1_500_001, -9_000, 16_384), (1_200_000, 0, 1_000_000),
                                       (2_000_001, 100, 4_096)])
def test_partitioned_shapes(gpu, preds, aggs, n, lo, span):
    """At least 2^20 rows over a direct array too large for shared memory:
    hot slots in shared memory, every other row an entry of its slot range's
    partition, then the partition pass (few partitions split into stripes,
    or many partitions with one owner each; sparse partitions update the
    records directly, dense ones -- span 4096 -- through a shared table)."""
    d = _data(n, seed=94 + n % 5, lo=lo, span=span)
    t = gpu.table(d)
    try:
        _same(_run(gpu, t, preds, aggs), _want(d, preds, aggs))
    finally:
        gpu.release(t)


def test_partitioned_zipf_keys(gpu):
    """Skewed keys: the hot cache takes the head, the partitions the tail."""
    from teide_b200 import workloads
    c = workloads.zipf_group_table(n=2_000_000, seed=95, nkeys=1 << 16)
    d = {"region": c["key"], "qty": c["v1"], "amount": c["v2"], "flag": (c["v1"] & 3)}
    t = gpu.table(d)
    try:
        preds = [("flag", "ne", 1)]
        _same(_run(gpu, t, preds, AGGS5), _want(d, preds, AGGS5))
    finally:
        gpu.release(t)


def test_partition_overflow_falls_back_to_atomics(gpu):
    """The sample reads every 4th row; keys that differ between sampled and
    unsampled rows make one key range's estimate far too small, so most of
    its rows overflow their regions and update the records directly."""
    n = 1_200_000
    r = np.random.default_rng(96)
    i = np.arange(n)
    key = np.where(i % 4 == 0, r.integers(0, 8192, n), r.integers(8192, 40_000, n)).astype(np.int64)
    d = {"flag": r.integers(0, 4, n, dtype=np.int64), "region": key,
         "amount": r.random(n) * 1000.0, "qty": r.integers(-500, 500, n, dtype=np.int64)}
    t = gpu.table(d)
    try:
        _same(_run(gpu, t, [], AGGS5), _want(d, [], AGGS5))
    finally:
        gpu.release(t)


def test_partition_long_runs(gpu):
    """About 2000 warm keys of ~400 rows each, more than the hot cache holds,
    over a sparse 1M-key range: the warm keys left out of the cache put long
    runs of one slot in otherwise sparse partitions, which then update the
    records directly instead of sorting their entries."""
    r = np.random.default_rng(97)
    n_warm, n_flat = 800_000, 400_000
    warm = r.choice(1_000_000, 2000, replace=False)
    key = np.concatenate([warm[r.integers(0, 2000, n_warm)], r.integers(0, 1_000_000, n_flat)]).astype(np.int64)
    r.shuffle(key)
    n = len(key)
    d = {"flag": r.integers(0, 4, n, dtype=np.int64), "region": key,
         "amount": r.standard_normal(n), "qty": r.integers(-10**12, 10**12, n, dtype=np.int64)}
    t = gpu.table(d)
    try:
        _same(_run(gpu, t, [("flag", "ne", 3)], AGGS5), _want(d, [("flag", "ne", 3)], AGGS5))
    finally:
        gpu.release(t)


def test_autotuned_launch_shape(gpu, tmp_path, monkeypatch):
    """A streaming group-by of 2^22 rows or more is first run once per
    candidate CTAs-per-SM value; the fastest is recorded in the tuner's JSON
    file under a "stream:" key and reused.  The tuned call and a later call
    of the same shape class both equal the oracle."""
    import json
    cache = tmp_path / "tune.json"
    monkeypatch.setenv("TD_TUNE_CACHE", str(cache))
    n = (1 << 22) + 6
    d = _data(n, 97, lo=-3, span=301)           # a shape class no other test in this file uses
    aggs = [(OP_SUM, "qty"), (OP_MIN, "amount"), (OP_MAX, "qty"), (OP_COUNT, "qty"), (OP_SUM, "amount")]
    tbl = gpu.table(d)
    first = _run(gpu, tbl, [("flag", "ne", 2)], aggs)
    entries = json.loads(cache.read_text())
    stream = {k: v for k, v in entries.items() if k.startswith("stream:")}
    assert len(stream) == 1 and list(stream.values())[0]["ctas_per_sm"] in (0, 1, 2, 4)
    again = _run(gpu, tbl, [("flag", "ne", 2)], aggs)
    gpu.release(tbl)
    _same(first, _want(d, [("flag", "ne", 2)], aggs))
    _same(again, _want(d, [("flag", "ne", 2)], aggs))
