"""The multi-GPU path's device half on one GPU: partial group-bys left on the
device by td_execute_device, and the merge of partial rows by the library's
own group-by (shard.merge_device, tdg_group_run on the device).

Three row shards stand for three ranks: each shard's partial result stays in
device memory, the partial rows are concatenated on the device (what the
all-gather of the exchange produces), and the merge must equal the oracle
over all rows -- integers exact, F64 within 1e-12 * max(|want|, sum |x|)."""
import ctypes as C

import numpy as np
import pytest
import torch

import oracle
from teide_b200 import shard, workloads
from teide_b200.pipelines import f64_tolerance_ok
from teide_b200.td import OP_AVG, OP_COUNT, OP_MAX, OP_MIN, OP_SUM

pytestmark = pytest.mark.gpu

AGGS = [(OP_COUNT, "v1"), (OP_SUM, "v1"), (OP_MIN, "v1"), (OP_MAX, "v1"), (OP_AVG, "v2")]


def _check(got, want, bounds):
    assert list(got) == list(want)
    for k in want:
        if k in bounds:
            assert f64_tolerance_ok(got[k], want[k], bounds[k]), k
        else:
            assert np.array_equal(got[k], want[k]), k


def _merged(gpu, parts_list, keys, aggs):
    parts, steps = shard.partial_plan(aggs)
    cat = {}
    for name in parts_list[0]:
        if name == "_result":
            continue
        cat[name] = torch.cat([p[name] for p in parts_list])
    out = shard.exchange_and_merge(cat, keys, parts, steps, device="cuda", td=gpu)
    for p in parts_list:
        gpu.release(p.pop("_result"))
    return out


@pytest.mark.parametrize("nkeys", [1 << 10, 1 << 20])
def test_device_partials_merge_to_the_whole_group_by(gpu, nkeys):
    c = workloads.zipf_group_table(n=600_000, seed=71, nkeys=nkeys)
    n = len(c["key"])
    parts, _ = shard.partial_plan(AGGS)
    shards = []
    for r in range(3):
        lo, hi = n * r // 3, n * (r + 1) // 3
        t = gpu.table({k: v[lo:hi] for k, v in c.items()})
        shards.append(shard.local_group(gpu, t, ("v1", "gt", 0), ["key"], parts))
        gpu.release(t)
    got = _merged(gpu, shards, ["key"], AGGS)
    m = c["v1"] > 0
    a = [(op, col, None if op == OP_COUNT else c[col]) for op, col in AGGS]
    _check(got, oracle.group({"key": c["key"]}, a, m), oracle.abs_bounds({"key": c["key"]}, a, m))


def test_device_partials_of_the_fused_join(gpu):
    b, p = workloads.join_tables(n_build=50_000, n_probe=900_000, seed=72)
    aggs = [(OP_SUM, "price"), (OP_COUNT, "price"), (OP_AVG, "price"), (OP_MAX, "qty")]
    parts, _ = shard.partial_plan(aggs)
    bt = gpu.table(b)
    n = len(p["fk"])
    shards = []
    for r in range(3):
        lo, hi = n * r // 3, n * (r + 1) // 3
        pt = gpu.table({k: v[lo:hi] for k, v in p.items()})
        shards.append(shard.local_join_group(gpu, bt, pt, ("qty", "gt", 10), "fk", "pk", ["cat"], parts))
        gpu.release(pt)
    gpu.release(bt)
    got = _merged(gpu, shards, ["cat"], aggs)
    j = oracle.join(p, b, ["fk"], ["pk"], 0, p["qty"] > 10)
    a = [(op, col, None if op == OP_COUNT else j[col]) for op, col in aggs]
    _check(got, oracle.group({"cat": j["cat"]}, a), oracle.abs_bounds({"cat": j["cat"]}, a))


def test_execute_device_then_fetch(gpu):
    """td_execute_device leaves the columns on the device; td_gpu_fetch
    brings the same values to the host elements."""
    c = workloads.readme_table(n=200_000, seed=73)
    t = gpu.table(c)
    g = gpu.graph(t)
    try:
        p = g.op("eq", g.scan("flag"), g.i64(0))
        root = g.group([g.filter(g.scan("region"), p)], [OP_SUM, OP_COUNT], [g.filter(g.scan("amount"), p)] * 2)
        part = shard._execute_device(gpu, g, root)
    finally:
        g.free()
    r = part.pop("_result")
    gpu.lib.td_gpu_fetch.argtypes = [C.c_void_p]
    assert gpu.lib.td_gpu_fetch(r) == 0
    host = gpu.table_dict(r)
    for k, v in part.items():
        assert np.array_equal(host[k], v.cpu().numpy()), k
    want = oracle.group({"region": c["region"]}, [(OP_SUM, "amount", c["amount"]), (OP_COUNT, "amount", None)],
                        c["flag"] == 0)
    assert np.array_equal(host["region"], want["region"]) and np.array_equal(host["amount_count"],
                                                                             want["amount_count"])
    gpu.release(r)
    gpu.release(t)
