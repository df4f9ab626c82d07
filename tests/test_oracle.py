"""Pins the numpy oracle (oracle/oracle.py) to Teide itself.

1. Against the committed golden fixtures, which hold Teide's own outputs
   (generated by tests/golden/make_golden.py from the compiled reference).
2. Against Teide's unit-test known answers.
3. Against the compiled reference run live on fresh seeded inputs (skipped
   where oracle/_ref/libteide_ref.so is not built).
"""
import os

import numpy as np
import pytest

import oracle
from teide_b200 import workloads
from teide_b200.td import OP_AVG, OP_COUNT, OP_MAX, OP_MIN, OP_SUM

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def load(name):
    with np.load(os.path.join(GOLD, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def pick(z, prefix):
    return {k[len(prefix):]: v for k, v in z.items() if k.startswith(prefix)}


def assert_group_equal(got, want, keys, ftol=1e-12):
    got = oracle.canonical(got, by=keys)
    want = oracle.canonical(want, by=keys)
    assert list(got) == list(want), (list(got), list(want))
    for k in want:
        g, w = np.asarray(got[k]), np.asarray(want[k])
        assert g.shape == w.shape, k
        if w.dtype.kind == "f":
            scale = np.maximum(np.abs(w), 1.0)
            assert np.all(np.abs(g - w) <= ftol * scale), k
        else:
            assert np.array_equal(g, w), k


def test_oracle_readme_golden():
    z = load("readme_small")
    cin = pick(z, "in_")
    m = oracle.conj(cin, [("flag", "eq", 0)])
    got = oracle.group({"region": cin["region"]}, [(OP_SUM, "amount", cin["amount"])], m)
    assert_group_equal(got, pick(z, "out_"), ["region"])


def test_oracle_zipf_group_golden():
    z = load("zipf_group_small")
    c = pick(z, "in_")
    m = oracle.conj(c, [("v1", "gt", 0)])
    got = oracle.group({"key": c["key"]}, [(OP_COUNT, "v1", None), (OP_SUM, "v1", c["v1"]),
                                           (OP_MIN, "v1", c["v1"]), (OP_MAX, "v1", c["v1"]),
                                           (OP_AVG, "v2", c["v2"])], m)
    assert_group_equal(got, pick(z, "out_"), ["key"])


def test_oracle_join_group_golden():
    z = load("join_group_small")
    b, p = pick(z, "b_"), pick(z, "p_")
    m = oracle.conj(p, [("qty", "gt", 10)])
    j = oracle.join(p, b, ["fk"], ["pk"], 0, m)
    assert oracle.canonical(j).keys() == pick(z, "join_").keys()
    for k, v in oracle.canonical(j).items():
        assert np.array_equal(v, pick(z, "join_")[k]), k
    got = oracle.group({"cat": j["cat"]}, [(OP_SUM, "price", j["price"]), (OP_COUNT, "price", None)])
    assert_group_equal(got, pick(z, "out_"), ["cat"])


@pytest.mark.parametrize("jt", [0, 1, 2])
def test_oracle_outer_join_golden(jt):
    z = load("join_outer_small")
    left, right = pick(z, "l_"), pick(z, "r_")
    got = oracle.canonical(oracle.join(left, right, ["id"], ["id"], jt))
    want = pick(z, f"j{jt}_")
    assert list(got) == list(want)
    for k in want:
        assert np.array_equal(got[k], want[k]), k


@pytest.mark.parametrize("case", ["a", "b", "c", "d"])
def test_oracle_sort_golden(case):
    """Teide's row order for a sort: I64 ties, F64 DESC with NaN and signed
    zeros (radix path), two keys with signed zeros (comparator), BOOL / I16 /
    U8 keys.  Bit-exact, F64 compared as bit patterns."""
    z = load("sort_small")
    cols = pick(z, case + "_in_")
    keys = []
    for spec in z[case + "_keys"]:
        name, desc, nf = str(spec).split(":")
        keys.append((name, bool(int(desc)), None if int(nf) < 0 else bool(int(nf))))
    got = oracle.sort(cols, keys)
    want = pick(z, case + "_out_")
    assert list(got) == list(want)
    for k in want:
        g, w = np.asarray(got[k]), np.asarray(want[k])
        if w.dtype == np.float64:
            g, w = g.view(np.uint64), w.view(np.uint64)
        assert np.array_equal(g.astype(w.dtype), w), (case, k)


def test_oracle_known_answers():
    id1 = np.array([1, 1, 2, 2, 3, 3, 1, 2, 3, 1])
    v1 = np.array([10, 20, 30, 40, 50, 60, 70, 80, 90, 100])
    cols = {"v1": v1}
    for op, n in {"eq": 1, "ne": 9, "lt": 4, "le": 5, "gt": 5, "ge": 6}.items():
        assert oracle.conj(cols, [("v1", op, 50)]).sum() == n
    g = oracle.group({"id1": id1}, [(OP_SUM, "v1", v1)])
    assert dict(zip(g["id1"], g["v1_sum"])) == {1: 200, 2: 150, 3: 200}
    i = np.arange(100_000)
    li, ri = oracle.join_pairs([i % 50000], [i % 50000])
    assert len(li) == 200_000 and (i * 10)[ri].sum() == 99_999_000_000
    li, ri = oracle.join_pairs([i[:80000]], [i[:80000] + 40000], 2)
    assert len(li) == 120_000
    li, ri = oracle.join_pairs([np.full(100_000, 42)], [i], 0)
    assert len(li) == 100_000 and ((i * 7)[ri] == 294).all()


def test_oracle_integer_sum_wraps():
    big = np.array([2**62, 2**62, 2**62, -5], np.int64)
    g = oracle.group({"k": np.zeros(4, np.int64)}, [(OP_SUM, "v", big)])
    with np.errstate(over="ignore"):
        assert g["v_sum"][0] == np.int64(2**62) * 3 - 5


# ---- live comparison with the compiled reference -----------------------------------

def _ref_group(ref, cols, pred, keys, aggs):
    import sys
    sys.path.insert(0, GOLD)
    from make_golden import ref_filter_group
    return ref_filter_group(ref, cols, pred, keys, aggs)


@pytest.mark.parametrize("seed", [7, 8])
def test_oracle_vs_reference_filter_group(ref, seed):
    c = workloads.zipf_group_table(n=60_000, seed=seed, nkeys=1 << 14)
    aggs = [(OP_COUNT, "v1"), (OP_SUM, "v1"), (OP_MIN, "v1"), (OP_MAX, "v1"), (OP_AVG, "v2")]
    want = _ref_group(ref, c, ("v1", "gt", 0), ["key"], aggs)
    m = oracle.conj(c, [("v1", "gt", 0)])
    got = oracle.group({"key": c["key"]}, [(a, nm, None if a == OP_COUNT else c[nm]) for a, nm in aggs], m)
    assert_group_equal(got, want, ["key"])


def test_oracle_vs_reference_filter_join_group(ref):
    import sys
    sys.path.insert(0, GOLD)
    from make_golden import ref_filter_join_group
    b, p = workloads.join_tables(n_build=20_000, n_probe=80_000, seed=9)
    want, joined = ref_filter_join_group(ref, b, p, ("qty", "gt", 10), "fk", "pk", ["cat"],
                                         [(OP_SUM, "price"), (OP_COUNT, "price")])
    m = oracle.conj(p, [("qty", "gt", 10)])
    j = oracle.join(p, b, ["fk"], ["pk"], 0, m)
    for k, v in oracle.canonical(j).items():
        assert np.array_equal(v, joined[k]), k
    got = oracle.group({"cat": j["cat"]}, [(OP_SUM, "price", j["price"]), (OP_COUNT, "price", None)])
    assert_group_equal(got, want, ["cat"])


# ---- the direct-array forms used by the full-size parity tests ---------------------

def test_group_direct_zipf_golden():
    """group_direct gives Teide's own output on the Zipf fixture."""
    z = load("zipf_group_small")
    c = pick(z, "in_")
    m = oracle.conj(c, [("v1", "gt", 0)])
    got = oracle.group_direct(c["key"], [(OP_COUNT, "v1", None), (OP_SUM, "v1", c["v1"]),
                                         (OP_MIN, "v1", c["v1"]), (OP_MAX, "v1", c["v1"]),
                                         (OP_AVG, "v2", c["v2"])], m)
    assert_group_equal(got, pick(z, "out_"), ["key"])


@pytest.mark.parametrize("seed", [0, 1])
def test_group_direct_equals_group(seed):
    r = np.random.default_rng(seed)
    n = 300_000
    k = r.integers(-5000, 70_000, n)
    vi = r.integers(-(2**62), 2**62, n)            # sums wrap
    vf = r.standard_normal(n)
    m = r.random(n) < 0.6
    aggs = [(OP_COUNT, "vi", None), (OP_SUM, "vi", vi), (OP_MIN, "vi", vi), (OP_MAX, "vi", vi),
            (OP_SUM, "vf", vf), (OP_AVG, "vf", vf), (OP_MIN, "vf", vf), (OP_MAX, "vf", vf)]
    want = oracle.group({"key": k}, aggs, m)
    got = oracle.group_direct(k, aggs, m)
    assert list(got) == list(want)
    for name in want:
        if want[name].dtype.kind == "f":
            assert np.allclose(got[name], want[name], rtol=1e-12, atol=1e-9), name
        else:
            assert np.array_equal(got[name], want[name]), name
    empty = oracle.group_direct(k, aggs, np.zeros(n, bool))
    assert all(len(v) == 0 for v in empty.values())


def test_join_unique_direct_golden():
    """join_unique_direct gives the same pairs as join_pairs and Teide's joined rows."""
    z = load("join_group_small")
    b, p = pick(z, "b_"), pick(z, "p_")
    m = oracle.conj(p, [("qty", "gt", 10)])
    li, ri = oracle.join_unique_direct(p["fk"], b["pk"], m)
    li2, ri2 = oracle.join_pairs([p["fk"]], [b["pk"]], 0, m)
    assert np.array_equal(li, li2) and np.array_equal(ri, ri2)
    j = {"fk": p["fk"][li], "qty": p["qty"][li], "price": p["price"][li], "cat": b["cat"][ri]}
    for k, v in oracle.canonical(j).items():
        assert np.array_equal(v, pick(z, "join_")[k]), k
    with pytest.raises(ValueError):
        oracle.join_unique_direct(np.arange(5), np.array([1, 2, 2]))
