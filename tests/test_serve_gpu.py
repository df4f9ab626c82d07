"""The request loop on the GPU: every result is the same alone and in the mix.

A scaled-down served mix (group table 3M rows of the Zipf-key shape, build
200K / probe 3M rows of the join shape, ranges of 10K..1M rows, random
thresholds) runs once query by query on the calling thread, then all at once
through a server with 8 slots.  Integer columns must match exactly and F64
columns within 1e-12 relative (their summation order depends on atomics).
A few requests are also checked against the oracle."""
import numpy as np
import pytest

import oracle
from teide_b200 import serve, workloads
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


def _same(a, b, what):
    assert list(a) == list(b), what
    for k in a:
        if a[k].dtype.kind == "f":
            assert np.allclose(a[k], b[k], rtol=1e-12, atol=1e-9, equal_nan=True), (what, k)
        else:
            assert np.array_equal(a[k], b[k]), (what, k)


def _canon(d, kind):
    return oracle.canonical(d, by=["key"] if kind == "group" else ["cat"])


def test_alone_equals_mix(tables):
    td, _, (tg, tb, tp) = tables
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
                _same(alone[i], _canon(td.table_dict(res), r.kind), f"request {i} ({r.kind})")
                td.release(res)
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
                sl = slice(r.off, r.off + r.n)
                if r.kind == "group":
                    m = c2["v1"][sl] > r.threshold
                    want = oracle.group({"key": c2["key"][sl]},
                                        [(OP_COUNT, "v1", None), (OP_SUM, "v1", c2["v1"][sl]),
                                         (OP_MIN, "v1", c2["v1"][sl]), (OP_MAX, "v1", c2["v1"][sl]),
                                         (OP_AVG, "v2", c2["v2"][sl])], mask=m)
                else:
                    left = {k: v[sl] for k, v in p.items()}
                    j = oracle.join(left, b, ["fk"], ["pk"], 0, lmask=left["qty"] > r.threshold)
                    want = oracle.group({"cat": j["cat"]}, [(OP_SUM, "price", j["price"]),
                                                            (OP_COUNT, "price", None)])
                _same(_canon(want, r.kind), got, f"{r.kind} [{r.off}, +{r.n}) t={r.threshold}")
    finally:
        serve.release(td, reqs)


def test_budget_serializes_and_stays_correct(tables):
    td, _, (tg, tb, tp) = tables
    reqs = _requests(10, seed=13)
    serve.build(td, reqs, tg, tb, tp)
    try:
        outs = []
        for slots, budget in ((8, 1), (8, 0)):
            with serve.Server(td, slots=slots, hbm_budget=budget) as s:
                ts = [s.submit(r.graph, r.root) for r in reqs]
                res = []
                for r, t in zip(reqs, ts):
                    p_, tm = s.wait(t)
                    assert tm.status == 0
                    res.append(_canon(td.table_dict(p_), r.kind))
                    td.release(p_)
                if budget == 1:
                    assert s.stats().peak_in_flight == 1
                outs.append(res)
        for i, (a, b_) in enumerate(zip(*outs)):
            _same(a, b_, f"request {i}")
    finally:
        serve.release(td, reqs)
