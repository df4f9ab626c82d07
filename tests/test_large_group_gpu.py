"""Large direct arrays (2^22 Zipf keys, 6M rows: global records with the
sampled hot-slot cache): parity with the oracle, with and without a filter."""
import numpy as np
import pytest

import oracle
from teide_b200.pipelines import readme_group
from teide_b200.td import OP_AVG, OP_COUNT, OP_MAX, OP_MIN, OP_SUM

pytestmark = pytest.mark.gpu

AGGS = [(OP_COUNT, "v1"), (OP_SUM, "v1"), (OP_MIN, "v1"), (OP_MAX, "v1"), (OP_AVG, "v2")]


def _plain_group(td, t):
    g = td.graph(t)
    try:
        r = g.execute(g.group([g.scan("key")], [a for a, _ in AGGS], [g.scan(n) for _, n in AGGS]))
    finally:
        g.free()
    out = td.table_dict(r)
    td.release(r)
    return out


def _want(c, mask=None):
    return oracle.group({"key": c["key"]}, [(op, n, None if op == OP_COUNT else c[n]) for op, n in AGGS], mask=mask)


def _check(got, want):
    assert list(got) == list(want)
    assert np.array_equal(got["key"], want["key"])
    for k in ("v1_count", "v1_sum", "v1_min", "v1_max"):
        assert np.array_equal(got[k], want[k]), k
    assert np.allclose(got["v2_mean"], want["v2_mean"], rtol=1e-12, atol=1e-12)


def _zipf_table(n, bits, seed):
    from teide_b200 import workloads
    c = workloads.zipf_group_table(n=n, seed=seed, nkeys=1 << bits)
    return c


@pytest.mark.parametrize("filtered", [False, True])
def test_large_direct_array_matches_oracle(gpu, filtered):
    c = _zipf_table(6_000_000, 22, seed=71)
    t = gpu.table(c)
    try:
        if filtered:
            got = readme_group(gpu, t, ("v1", "gt", 0), ["key"], AGGS)
            want = _want(c, c["v1"] > 0)
        else:
            got = _plain_group(gpu, t)
            want = _want(c)
        _check(got, want)
    finally:
        gpu.release(t)
