"""td_execute_batch: many group-by graphs in one launch (the batched-query shape:
thousands of small SUM/COUNT/MAX-by-key queries over resident tables).

Each query's rows in the packed result must equal the oracle's group-by of
that query's table (keys, COUNT exact; SUM/MAX of F64 within 1e-12), and a
repeated call -- which replays the cached CUDA graph -- must return the same
rows."""
import ctypes as C

import numpy as np
import pytest

import oracle
from teide_b200 import workloads
from teide_b200.pipelines import f64_tolerance_ok
from teide_b200.td import OP_COUNT, OP_MAX, OP_SUM

pytestmark = pytest.mark.gpu


def _bind(td):
    L = td.lib
    L.td_execute_batch.restype = C.c_void_p
    L.td_execute_batch.argtypes = [C.c_void_p, C.c_void_p, C.c_int64]
    L.td_gpu_pin.argtypes = [C.c_void_p]
    return L


def run_batch(td, tables, ops=(OP_SUM, OP_COUNT, OP_MAX)):
    L = _bind(td)
    graphs, roots = [], []
    for t in tables:
        g = td.graph(t)
        roots.append(g.group([g.scan("key")], list(ops), [g.scan("val")] * len(ops)))
        graphs.append(g)
    G = (C.c_void_p * len(graphs))(*[g.g for g in graphs])
    R = (C.c_void_p * len(roots))(*roots)
    r = td.check(L.td_execute_batch(G, R, len(graphs)), "batch")
    out = td.table_dict(r)
    td.release(r)
    for g in graphs:
        g.free()
    return out


def test_batch_matches_oracle_per_query(gpu, tmp_path, monkeypatch):
    monkeypatch.setenv("TD_TUNE_CACHE", str(tmp_path / "tune.json"))
    # 300 queries: the batch runs as 4 chunks whose results are copied while later chunks compute
    rows, ks = workloads.batch_shapes(n_queries=300, seed=41, rows=(1, 200_000), groups=(1, 70_000))
    datas = [workloads.batch_query(int(r), int(k), seed=1000 + i) for i, (r, k) in enumerate(zip(rows, ks))]
    tables = [gpu.table(d) for d in datas]
    L = _bind(gpu)
    for t in tables:
        assert L.td_gpu_pin(t) == 0
    first = run_batch(gpu, tables)
    again = run_batch(gpu, tables)                   # cached graph replay
    assert list(first) == ["_query", "key", "val_sum", "val_count", "val_max"]
    for name in ("_query", "key", "val_count", "val_max"):
        assert np.array_equal(first[name], again[name]), name
    # F64 sums: within 1e-12 * sum |val| of the group (val >= 0, so of the sum itself)
    assert f64_tolerance_ok(first["val_sum"], again["val_sum"], np.abs(again["val_sum"]) * 2)
    q = first["_query"]
    assert np.all(np.diff(q) >= 0)                    # grouped by query, in order
    for i, d in enumerate(datas):
        sel = q == i
        want = oracle.group({"key": d["key"]}, [(OP_SUM, "val", d["val"]), (OP_COUNT, "val", None),
                                                (OP_MAX, "val", d["val"])])
        assert np.array_equal(first["key"][sel], want["key"]), i
        assert np.array_equal(first["val_count"][sel], want["val_count"]), i
        absum = oracle.group({"key": d["key"]}, [(OP_SUM, "val", np.abs(d["val"]))])["val_sum"]
        assert f64_tolerance_ok(first["val_sum"][sel], want["val_sum"], absum), i
        assert np.array_equal(first["val_max"][sel], want["val_max"]), i
    for t in tables:
        gpu.release(t)


def test_batch_rejects_mixed_shapes(gpu):
    a = gpu.table({"key": np.arange(10, dtype=np.int64), "val": np.ones(10)})
    b = gpu.table({"key": np.arange(10, dtype=np.int64), "val": np.ones(10)})
    L = _bind(gpu)
    ga, gb = gpu.graph(a), gpu.graph(b)
    ra = ga.group([ga.scan("key")], [OP_SUM], [ga.scan("val")])
    rb = gb.group([gb.scan("key")], [OP_MAX], [gb.scan("val")])
    G = (C.c_void_p * 2)(ga.g, gb.g)
    R = (C.c_void_p * 2)(ra, rb)
    p = L.td_execute_batch(G, R, 2) or 0
    assert p == 7                                     # TD_ERR_NYI
    ga.free(); gb.free()
    gpu.release(a); gpu.release(b)


def test_batch_equals_per_query_execute_narrow_types(gpu):
    """I32 keys and I32 values: keys and MIN/MAX come back as I32, SUM as I64,
    AVG as F64 -- the same columns td_execute returns for each graph."""
    from teide_b200.td import I32, OP_AVG, OP_MIN
    r = np.random.default_rng(7)
    datas = []
    for i in range(20):
        n = int(r.integers(0, 50_000))
        lo = int(r.integers(-1000, 1000))
        datas.append({"key": (r.integers(lo, lo + int(r.integers(1, 3000)), n).astype(np.int32), I32),
                      "val": (r.integers(-2**31, 2**31 - 1, n).astype(np.int32), I32)})
    tables = [gpu.table(d) for d in datas]
    ops = (OP_SUM, OP_MIN, OP_MAX, OP_AVG, OP_COUNT)
    got = run_batch(gpu, tables, ops)
    q = got["_query"]
    for i, t in enumerate(tables):
        g = gpu.graph(t)
        root = g.group([g.scan("key")], list(ops), [g.scan("val")] * len(ops))
        p = g.execute(root, optimize=False)
        want = gpu.table_dict(p)
        gpu.release(p)
        g.free()
        sel = q == i
        for name, col in want.items():
            assert got[name].dtype == col.dtype, name
            if col.dtype.kind == "f":
                assert np.allclose(got[name][sel], col, rtol=1e-12), (i, name)
            else:
                assert np.array_equal(got[name][sel], col), (i, name)
    for t in tables:
        gpu.release(t)


@pytest.mark.parametrize("ctas", [1, 0])
def test_batch_key_slices(gpu, tmp_path, monkeypatch, ctas):
    """Queries whose key range exceeds shared memory but has at least 8 rows
    per slot are aggregated by key slice (an item is a (tile, slice) pair):
    with one CTA per SM (about 11K slots on chip) the 30000- and 15000-slot
    queries take 3 and 2 slices; with the default 48 KB (about 2.4K slots) the
    15000-slot one takes 7 and the 30000-slot one (13 would be needed) the
    global records.  The launch shape is fixed through the tuner's file.
    Every query equals the oracle's group-by."""
    import json
    import math
    specs = [(30000, 300_000), (15000, 200_000), (5000, 60_000), (100, 50_000), (30000, 250_000),
             (15000, 130_000), (2500, 40_000), (60, 10_000)]
    r = np.random.default_rng(400 + ctas)
    datas = []
    for k, n in specs:
        key = r.integers(0, k, n, dtype=np.int64)
        key[0], key[1] = 0, k - 1                        # the key range is exactly [0, k)
        datas.append({"key": key, "val": r.random(n) * 100.0})
    nq = len(specs)
    tkey = "batch:q%d:r%d:s%d:a%d" % (int(math.log2(nq)), int(math.log2(sum(n for _, n in specs) / nq)),
                                      int(math.log2(sum(k for k, _ in specs) / nq)), 3)
    cache = tmp_path / "tune.json"
    # the tuner's file format: one JSON object, one entry per line
    cache.write_text('{\n  "%s": {"tile_rows": 16384, "ctas_per_sm": %d}\n}\n' % (tkey, ctas))
    assert json.loads(cache.read_text())[tkey]["ctas_per_sm"] == ctas
    monkeypatch.setenv("TD_TUNE_CACHE", str(cache))
    tables = [gpu.table(d) for d in datas]
    L = _bind(gpu)
    for t in tables:
        assert L.td_gpu_pin(t) == 0
    try:
        got = run_batch(gpu, tables)
        q = got["_query"]
        for i, d in enumerate(datas):
            sel = q == i
            want = oracle.group({"key": d["key"]}, [(OP_SUM, "val", d["val"]), (OP_COUNT, "val", None),
                                                    (OP_MAX, "val", d["val"])])
            assert np.array_equal(got["key"][sel], want["key"]), i
            assert np.array_equal(got["val_count"][sel], want["val_count"]), i
            assert np.array_equal(got["val_max"][sel], want["val_max"]), i
            assert f64_tolerance_ok(got["val_sum"][sel], want["val_sum"], np.abs(want["val_sum"])), i
    finally:
        for t in tables:
            gpu.release(t)
