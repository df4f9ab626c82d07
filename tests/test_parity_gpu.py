"""Parity of the GPU path with the oracle and with Teide's own outputs.

Integer results (keys, counts, integer sums, MIN/MAX, join rows) must be
bit-exact; F64 SUM/AVG must satisfy |got - want| <= 1e-12 * max(|want|,
sum |x|) per group (the summation order differs from the CPU's).  Every
case compares whole results, the two headline workloads at their stated
sizes (config 2: 200M rows; config 3: a 100M-row probe) included.
"""
import os

import numpy as np
import pytest

import oracle
from teide_b200.pipelines import (f64_tolerance_ok, fused_join_group, join_then_group, readme_group,
                           two_graph_group)
from teide_b200 import workloads
from teide_b200.td import OP_AVG, OP_COUNT, OP_MAX, OP_MIN, OP_SUM

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(__file__), "golden")
REL = 1e-12


def load(name):
    with np.load(os.path.join(GOLD, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def pick(z, prefix):
    return {k[len(prefix):]: v for k, v in z.items() if k.startswith(prefix)}


def check_group(got, want, keys, abs_sums=None):
    got = oracle.canonical(got, by=keys)
    want = oracle.canonical(want, by=keys)
    assert list(got) == list(want), (list(got), list(want))
    for k, w in want.items():
        g = np.asarray(got[k])
        assert g.dtype == w.dtype and g.shape == w.shape, (k, g.dtype, w.dtype, g.shape, w.shape)
        if w.dtype.kind == "f":
            a = abs_sums.get(k, np.abs(w)) if abs_sums else np.abs(w)
            assert f64_tolerance_ok(g, w, a, REL), (k, np.max(np.abs(g - w)))
        else:
            assert np.array_equal(g, w), k


def abs_sums_of(keys_d, vals, mask, name, suffix):
    g = oracle.group(keys_d, [(OP_SUM, name, np.abs(vals))], mask)
    return {name + suffix: g[name + "_sum"]}


C2_AGGS = [(OP_COUNT, "v1"), (OP_SUM, "v1"), (OP_MIN, "v1"), (OP_MAX, "v1"), (OP_AVG, "v2")]


def oracle_c2(c, mask):
    return oracle.group({"key": c["key"]}, [(a, n, None if a == OP_COUNT else c[n]) for a, n in C2_AGGS], mask)


# ---- golden fixtures (Teide's own outputs) -------------------------------------------

@pytest.mark.parametrize("form", ["readme", "two_graph"])
def test_readme_golden(gpu, form):
    z = load("readme_small")
    c = pick(z, "in_")
    t = gpu.table(c)
    fn = readme_group if form == "readme" else two_graph_group
    got = fn(gpu, t, ("flag", "eq", 0), ["region"], [(OP_SUM, "amount")])
    gpu.release(t)
    m = c["flag"] == 0
    check_group(got, pick(z, "out_"), ["region"], abs_sums_of({"region": c["region"]}, c["amount"], m, "amount", "_sum"))


@pytest.mark.parametrize("form", ["readme", "two_graph"])
def test_zipf_group_golden(gpu, form):
    z = load("zipf_group_small")
    c = pick(z, "in_")
    t = gpu.table(c)
    fn = readme_group if form == "readme" else two_graph_group
    got = fn(gpu, t, ("v1", "gt", 0), ["key"], C2_AGGS)
    gpu.release(t)
    m = c["v1"] > 0
    a = oracle.group({"key": c["key"]}, [(OP_SUM, "v2", np.abs(c["v2"]))], m)["v2_sum"]
    cnt = oracle.group({"key": c["key"]}, [(OP_COUNT, "v2", None)], m)["v2_count"]
    check_group(got, pick(z, "out_"), ["key"], {"v2_mean": a / cnt})


@pytest.mark.parametrize("form", ["fused", "two_call"])
def test_join_group_golden(gpu, form):
    z = load("join_group_small")
    b, p = pick(z, "b_"), pick(z, "p_")
    bt, pt = gpu.table(b), gpu.table(p)
    aggs = [(OP_SUM, "price"), (OP_COUNT, "price")]
    if form == "fused":
        got = fused_join_group(gpu, bt, pt, ("qty", "gt", 10), "fk", "pk", ["cat"], aggs)
    else:
        got, joined = join_then_group(gpu, bt, pt, ("qty", "gt", 10), "fk", "pk", ["cat"], aggs)
        want_j = pick(z, "join_")
        joined = oracle.canonical(joined)
        assert list(joined) == list(want_j)
        for k in want_j:
            assert np.array_equal(joined[k], want_j[k]), k
    gpu.release(bt)
    gpu.release(pt)
    m = oracle.conj(p, [("qty", "gt", 10)])
    j = oracle.join(p, b, ["fk"], ["pk"], 0, m)
    check_group(got, pick(z, "out_"), ["cat"], abs_sums_of({"cat": j["cat"]}, j["price"], None, "price", "_sum"))


@pytest.mark.parametrize("jt", [0, 1, 2])
def test_outer_join_golden(gpu, jt):
    z = load("join_outer_small")
    lt, rt = gpu.table(pick(z, "l_")), gpu.table(pick(z, "r_"))
    g = gpu.graph(lt)
    k = g.scan("id")
    r = g.execute(g.join(g.const_table(lt), [k], g.const_table(rt), [k], jt))
    g.free()
    got = oracle.canonical(gpu.table_dict(r))
    want = pick(z, f"j{jt}_")
    assert list(got) == list(want)
    for name in want:
        assert np.array_equal(got[name], want[name]), name
    for x in (r, lt, rt):
        gpu.release(x)


# ---- seeded cases against the oracle ---------------------------------------------------------

@pytest.mark.parametrize("n,nkeys,seed", [(1, 16, 1), (1000, 1 << 10, 2), (250_000, 1 << 16, 3),
                                          (2_000_000, 1 << 24, 4)])
def test_zipf_group_shapes_vs_oracle(gpu, n, nkeys, seed):
    c = workloads.zipf_group_table(n=n, seed=seed, nkeys=nkeys)
    t = gpu.table(c)
    got = readme_group(gpu, t, ("v1", "gt", 0), ["key"], C2_AGGS)
    gpu.release(t)
    m = c["v1"] > 0
    want = oracle_c2(c, m)
    a = oracle.group({"key": c["key"]}, [(OP_SUM, "v2", np.abs(c["v2"]))], m)["v2_sum"]
    cnt = want["v1_count"]
    check_group(got, want, ["key"], {"v2_mean": a / np.maximum(cnt, 1)})


def test_group_hash_path_wide_keys(gpu):
    """Keys spread over a range far wider than the row count take the hash
    table; F64 keys too."""
    r = np.random.default_rng(11)
    n = 300_000
    key = r.integers(-2**62, 2**62, 5000)[r.integers(0, 5000, n)]
    fkey = np.round(r.standard_normal(n) * 50) / 4
    v = r.integers(-1000, 1000, n)
    t = gpu.table({"k": key, "f": fkey, "v": v})
    for kname in ("k", "f"):
        g = gpu.graph(t)
        res = g.execute(g.group([g.scan(kname)], [OP_SUM, OP_MIN, OP_MAX, OP_COUNT],
                                [g.scan("v")] * 4))
        g.free()
        got = gpu.table_dict(res)
        gpu.release(res)
        kv = key if kname == "k" else fkey
        want = oracle.group({kname: kv}, [(OP_SUM, "v", v), (OP_MIN, "v", v), (OP_MAX, "v", v),
                                          (OP_COUNT, "v", None)])
        check_group(got, want, [kname])
    gpu.release(t)


def test_multi_key_group(gpu):
    r = np.random.default_rng(12)
    n = 200_000
    c = {"a": r.integers(0, 7, n), "b": r.integers(-3, 40, n), "x": r.random(n)}
    t = gpu.table(c)
    g = gpu.graph(t)
    res = g.execute(g.group([g.scan("a"), g.scan("b")], [OP_SUM, OP_AVG, OP_MAX], [g.scan("x")] * 3))
    g.free()
    got = gpu.table_dict(res)
    gpu.release(res)
    gpu.release(t)
    want = oracle.group({"a": c["a"], "b": c["b"]}, [(OP_SUM, "x", c["x"]), (OP_AVG, "x", c["x"]),
                                                     (OP_MAX, "x", c["x"])])
    check_group(got, want, ["a", "b"])


def test_readme_full_size(gpu):
    c = workloads.readme_table(n=10_000_000, seed=21)
    t = gpu.table(c)
    got = readme_group(gpu, t, ("flag", "eq", 0), ["region"], [(OP_SUM, "amount")])
    gpu.release(t)
    m = c["flag"] == 0
    want = oracle.group({"region": c["region"]}, [(OP_SUM, "amount", c["amount"])], m)
    check_group(got, want, ["region"], abs_sums_of({"region": c["region"]}, c["amount"], m, "amount", "_sum"))


def test_join_group_medium_vs_oracle(gpu):
    b, p = workloads.join_tables(n_build=1_000_000, n_probe=10_000_000, seed=22)
    bt, pt = gpu.table(b), gpu.table(p)
    aggs = [(OP_SUM, "price"), (OP_COUNT, "price")]
    got = fused_join_group(gpu, bt, pt, ("qty", "gt", 10), "fk", "pk", ["cat"], aggs)
    gpu.release(bt)
    gpu.release(pt)
    m = p["qty"] > 10
    j = oracle.join(p, b, ["fk"], ["pk"], 0, m)
    want = oracle.group({"cat": j["cat"]}, [(OP_SUM, "price", j["price"]), (OP_COUNT, "price", None)])
    check_group(got, want, ["cat"], abs_sums_of({"cat": j["cat"]}, j["price"], None, "price", "_sum"))


@pytest.mark.parametrize("jt", [1, 2])
def test_fused_outer_join_group(gpu, jt):
    """Outer joins feed zero-filled values of the missing side to the group-by,
    exactly as the materialized outer join would."""
    z = load("join_outer_small")
    left, right = pick(z, "l_"), pick(z, "r_")
    lt, rt = gpu.table(left), gpu.table(right)
    aggs = [(OP_SUM, "score"), (OP_COUNT, "score"), (OP_SUM, "val")]
    got = fused_join_group(gpu, rt, lt, ("val", "ge", -1000), "id", "id", ["id"], aggs, jt)
    gpu.release(lt)
    gpu.release(rt)
    j = oracle.join(left, right, ["id"], ["id"], jt)
    want = oracle.group({"id": j["id"]}, [(OP_SUM, "score", j["score"]), (OP_COUNT, "score", None),
                                          (OP_SUM, "val", j["val"])])
    check_group(got, want, ["id"])


def test_join_group_full_size_per_group(gpu):
    """Config 3 at its stated size (build 10M, probe 100M): every one of the
    1000 `cat` groups against the oracle -- COUNT bit-exact, SUM(price)
    within 1e-12 * max(|ref|, sum |price|) of the group."""
    b, p = workloads.join_tables(seed=23)
    bt, pt = gpu.table(b), gpu.table(p)
    got = fused_join_group(gpu, bt, pt, ("qty", "gt", 10), "fk", "pk", ["cat"],
                           [(OP_SUM, "price"), (OP_COUNT, "price")])
    gpu.release(bt)
    gpu.release(pt)
    li, ri = oracle.join_unique_direct(p["fk"], b["pk"], p["qty"] > 10)
    cat, price = b["cat"][ri], p["price"][li]
    del li, ri
    want = oracle.group_direct(cat, [(OP_SUM, "price", price), (OP_COUNT, "price", None)], key_name="cat")
    absum = oracle.group_direct(cat, [(OP_SUM, "price", np.abs(price))], key_name="cat")["price_sum"]
    assert len(want["cat"]) == 1000
    check_group(got, want, ["cat"], {"price_sum": absum})


def test_zipf_group_full_size_per_group(gpu):
    """Config 2 at its stated size (200M rows, Zipf(1.1) over 2^24 keys,
    filter v1 > 0): all ~5.9M groups against the oracle -- keys, COUNT,
    SUM, MIN and MAX of v1 bit-exact, AVG(v2) within 1e-12 * sum |v2| /
    count of the group."""
    c = workloads.zipf_group_table(n=200_000_000, seed=24, device="cuda")
    t = gpu.table(c)
    got = readme_group(gpu, t, ("v1", "gt", 0), ["key"], C2_AGGS)
    gpu.release(t)
    m = c["v1"] > 0
    want = oracle.group_direct(c["key"], [(a, n, None if a == OP_COUNT else c[n]) for a, n in C2_AGGS], m)
    abs_mean = oracle.group_direct(c["key"], [(OP_AVG, "v2", np.abs(c["v2"]))], m)["v2_mean"]
    assert len(want["key"]) > 5_000_000
    check_group(got, want, ["key"], {"v2_mean": abs_mean})
