"""The fused join probe's vector form and its fallbacks: odd probe lengths
(the last pair is half full), a probe view starting at an odd row (columns
not 16-byte aligned: the general kernel runs), COUNT only, no filter and two
filter terms -- each against the oracle."""
import numpy as np
import pytest

import oracle
from teide_b200.pipelines import const, f64_tolerance_ok
from teide_b200 import serve, workloads
from teide_b200.td import OP_COUNT, OP_MAX, OP_SUM

pytestmark = pytest.mark.gpu


def _run(td, build_t, probe_t, preds, aggs):
    g = td.graph(None)
    try:
        p = None
        for c, op, k in preds:
            q = g.op(op, g.scan(c), const(g, k))
            p = q if p is None else g.op("and", p, q)
        left = g.const_table(probe_t) if p is None else g.filter(g.const_table(probe_t), p)
        g.join(left, [g.scan("fk")], g.const_table(build_t), [g.scan("pk")], 0)
        r = td.check(td.lib.td_execute(g.g, g.group([g.scan("cat")], [a for a, _ in aggs],
                                                    [g.scan(n) for _, n in aggs])), "execute")
    finally:
        g.free()
    out = td.table_dict(r)
    td.release(r)
    return out


def _want(b, p, preds, aggs):
    m = np.ones(len(p["fk"]), bool)
    for c, op, k in preds:
        m &= oracle.compare(op, p[c], k)
    j = oracle.join(p, b, ["fk"], ["pk"], 0, lmask=m)
    keys = {"cat": j["cat"]}
    a = [(op, n, None if op == OP_COUNT else j[n]) for op, n in aggs]
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
    ([("qty", "gt", 10)], [(OP_SUM, "price"), (OP_COUNT, "price")]),
    ([], [(OP_COUNT, "price")]),
    ([], [(OP_SUM, "price"), (OP_MAX, "price")]),
    ([("qty", "gt", 10), ("qty", "lt", 90)], [(OP_COUNT, "qty")]),
    ([("qty", "gt", 10), ("price", "lt", 300.0)], [(OP_SUM, "price"), (OP_COUNT, "price")]),
    ([("qty", "ge", 50)], [(OP_SUM, "qty"), (OP_MAX, "qty"), (OP_COUNT, "qty")]),
]


@pytest.mark.parametrize("preds,aggs", CASES)
@pytest.mark.parametrize("n_probe", [300_001, 300_000])
def test_vector_probe_shapes(gpu, preds, aggs, n_probe):
    b, p = workloads.join_tables(n_build=50_000, n_probe=n_probe, seed=81)
    bt, pt = gpu.table(b), gpu.table(p)
    try:
        _same(_run(gpu, bt, pt, preds, aggs), _want(b, p, preds, aggs))
    finally:
        gpu.release(bt)
        gpu.release(pt)


def test_unaligned_probe_view_falls_back(gpu):
    b, p = workloads.join_tables(n_build=50_000, n_probe=200_000, seed=82)
    bt, pt = gpu.table(b), gpu.table(p)
    view = serve.table_slice(gpu, pt, 1, 150_001)          # starts 8 bytes into each column
    try:
        preds, aggs = CASES[0]
        sub = {k: v[1:150_002] for k, v in p.items()}
        _same(_run(gpu, bt, view, preds, aggs), _want(b, sub, preds, aggs))
    finally:
        gpu.release(view)
        gpu.release(bt)
        gpu.release(pt)


@pytest.mark.parametrize("n_build", [50_000, 50_003, 7])
def test_dense_build_keys_with_a_repeat(gpu, n_build):
    """Build keys spanning exactly as many values as there are build rows are
    written with plain stores and then checked for empty map entries: one key
    written twice leaves one entry empty, and the query must then give the
    join's true multiplicity (the general join), equal to the oracle's.  The
    odd sizes reach the hole check's tail entries; without the repeat the
    map path runs and must agree too."""
    b, p = workloads.join_tables(n_build=n_build, n_probe=200_001, seed=83)
    preds, aggs = CASES[0]
    for repeat in (False, True):
        bb = dict(b)
        if repeat:
            pk = bb["pk"].copy()
            pk[pk == n_build - 2] = 1                   # min 0 and max n-1 stay: the span is still n_build
            assert pk.min() == 0 and pk.max() == n_build - 1 and len(np.unique(pk)) == n_build - 1
            bb["pk"] = pk
        bt, pt = gpu.table(bb), gpu.table(p)
        try:
            _same(_run(gpu, bt, pt, preds, aggs), _want(bb, p, preds, aggs))
        finally:
            gpu.release(bt)
            gpu.release(pt)
