"""Sort / top-N cases shared by the reference pin (test_sort_ref.py, Teide on
the CPU) and the GPU parity tests (test_sort_gpu.py).  Each case builds its
table in the given library, runs td_sort_op (optionally under td_head)
through td_execute and returns (got, want): the result as {name: numpy}
(SYM columns as strings, F64 columns as bit patterns so NaN compares) and
the oracle's answer in the same form."""
import numpy as np

import oracle
from teide_b200.td import BOOL, I16, I32, OP_SUM, U8

ROWS = 3000


def _bits(d):
    return {k: (v.view(np.uint64) if isinstance(v, np.ndarray) and v.dtype == np.float64 else v)
            for k, v in d.items()}


def _strings(td, out, col):
    u, inv = np.unique(out[col], return_inverse=True)
    out[col] = np.array([td.sym_name(int(x)) for x in u], dtype=object)[inv]
    return out


def _run(td, tbl, keys, limit=None, sym=None):
    """keys: [(name, desc, nulls_first or None)]."""
    g = td.graph(tbl)
    try:
        t = g.const_table(tbl)
        nf = None if all(k[2] is None for k in keys) else [int(k[1] if k[2] is None else k[2]) for k in keys]
        root = g.sort(t, [g.scan(k[0]) for k in keys], [int(k[1]) for k in keys], nf)
        if limit is not None:
            root = g.head(root, limit)
        r = g.execute(root, optimize=False)
    finally:
        g.free()
    out = td.table_dict(r)
    td.release(r)
    if sym:
        out = _strings(td, out, sym)
    return out


def i64_ties(td, seed=1, n=ROWS):
    """One I64 key with many equal values: equal keys keep their row order."""
    r = np.random.default_rng(seed)
    d = {"k": r.integers(0, 50, n), "i": np.arange(n), "v": r.standard_normal(n)}
    t = td.table(d)
    try:
        keys = [("k", False, None)]
        return _bits(_run(td, t, keys)), _bits(oracle.sort(d, keys))
    finally:
        td.release(t)


def f64_desc_nan_zero(td, seed=2, n=2000):
    """F64 DESC with NaN (first, the DESC default), -0.0 / +0.0 and repeats."""
    r = np.random.default_rng(seed)
    f = np.round(r.standard_normal(n), 1)
    f[r.integers(0, n, 40)] = np.nan
    f[r.integers(0, n, 40)] = -0.0
    f[r.integers(0, n, 40)] = 0.0
    d = {"f": f, "i": np.arange(n)}
    t = td.table(d)
    try:
        keys = [("f", True, None)]
        return _bits(_run(td, t, keys)), _bits(oracle.sort(d, keys))
    finally:
        td.release(t)


def f64_asc_nan_first(td, seed=3, n=1500):
    """F64 ascending with NaN placed first."""
    r = np.random.default_rng(seed)
    f = r.standard_normal(n)
    f[r.integers(0, n, 30)] = np.nan
    d = {"f": f, "i": np.arange(n)}
    t = td.table(d)
    try:
        keys = [("f", False, True)]
        return _bits(_run(td, t, keys)), _bits(oracle.sort(d, keys))
    finally:
        td.release(t)


def i32_key(td, seed=4, n=ROWS):
    r = np.random.default_rng(seed)
    d = {"k": r.integers(-2**31, 2**31 - 1, n).astype(np.int32), "i": np.arange(n)}
    t = td.table({"k": (d["k"], I32), "i": d["i"]})
    try:
        keys = [("k", False, None)]
        return _run(td, t, keys), oracle.sort(d, keys)
    finally:
        td.release(t)


def two_keys(td, seed=5, n=2500):
    """I64 ascending, then I32 descending; ties on both keep row order."""
    r = np.random.default_rng(seed)
    d = {"a": r.integers(0, 10, n), "b": r.integers(-5, 5, n).astype(np.int32), "i": np.arange(n)}
    t = td.table({"a": d["a"], "b": (d["b"], I32), "i": d["i"]})
    try:
        keys = [("a", False, None), ("b", True, None)]
        return _run(td, t, keys), oracle.sort(d, keys)
    finally:
        td.release(t)


def sym_key(td, seed=6, n=1500):
    """SYM key ordered by its strings ("w10" before "w2")."""
    r = np.random.default_rng(seed)
    words = [f"w{i}" for i in range(200)]
    ids = np.array([td.sym(w) for w in words], dtype=np.int64)
    pick = r.integers(0, 200, n)
    sv = td.sym_vec(ids[pick], 3)
    t = td.table({"s": sv, "i": np.arange(n)})
    td.release(sv)
    try:
        keys = [("s", False, None)]
        want = oracle.sort({"s": np.array(words, dtype=object)[pick], "i": np.arange(n)}, keys)
        return _run(td, t, keys, sym="s"), want
    finally:
        td.release(t)


def head_of_sort(td, seed=7, n=5000, limit=10):
    """Top 10 of unique keys, DESC (Teide's heap top-N path)."""
    r = np.random.default_rng(seed)
    d = {"k": r.permutation(n).astype(np.int64) * 7 - 1000, "v": r.standard_normal(n)}
    t = td.table(d)
    try:
        keys = [("k", True, None)]
        return _bits(_run(td, t, keys, limit=limit)), _bits(oracle.sort(d, keys, limit))
    finally:
        td.release(t)


def sort_of_group(td, seed=8, n=20_000):
    """Group-by result sorted by its SUM, descending."""
    r = np.random.default_rng(seed)
    d = {"k": r.integers(0, 300, n), "v": r.integers(-1000, 1000, n)}
    t = td.table(d)
    try:
        g = td.graph(t)
        try:
            grp = g.group([g.scan("k")], [OP_SUM], [g.scan("v")])
            root = g.sort(grp, [g.scan("v_sum")], [1])
            res = g.execute(root, optimize=False)
        finally:
            g.free()
        got = td.table_dict(res)
        td.release(res)
        grouped = oracle.group({"k": d["k"]}, [(OP_SUM, "v", d["v"])])
        return got, oracle.sort(grouped, [("v_sum", True, None)])
    finally:
        td.release(t)


def small_int_keys(td, seed=9, n=ROWS):
    """BOOL ascending, I16 descending, U8 ascending (Teide's comparator sort:
    unsigned bytes, signed 16-bit), with F64 ±0.0 carried along."""
    r = np.random.default_rng(seed)
    d = {"b": r.integers(0, 2, n).astype(np.bool_), "h": r.integers(-300, 300, n).astype(np.int16),
         "u": r.integers(0, 256, n).astype(np.uint8), "f": np.where(r.integers(0, 2, n) == 1, -0.0, 0.0),
         "i": np.arange(n)}
    t = td.table({"b": (d["b"], BOOL), "h": (d["h"], I16), "u": (d["u"], U8), "f": d["f"], "i": d["i"]})
    try:
        keys = [("b", False, None), ("h", True, None), ("u", False, None)]
        return _bits(_run(td, t, keys)), _bits(oracle.sort(d, keys))
    finally:
        td.release(t)


def f64_zeros_two_keys(td, seed=10, n=ROWS):
    """F64 key holding -0.0 and +0.0, then an I64 key: the zeros compare
    equal (the composite does not fit 64 bits, Teide's comparator decides)."""
    r = np.random.default_rng(seed)
    f = np.round(r.standard_normal(n), 0)
    f[r.integers(0, n, 600)] = -0.0
    f[r.integers(0, n, 600)] = 0.0
    d = {"f": f, "k": r.integers(0, 5, n), "i": np.arange(n)}
    t = td.table(d)
    try:
        keys = [("f", True, None), ("k", False, None)]
        return _bits(_run(td, t, keys)), _bits(oracle.sort(d, keys))
    finally:
        td.release(t)


def f64_zeros_small(td, seed=11, n=50):
    """At most 64 rows Teide sorts by insertion with its comparator: -0.0
    equals +0.0, NaN last."""
    r = np.random.default_rng(seed)
    f = np.where(r.integers(0, 2, n) == 1, -0.0, 0.0)
    f[r.integers(0, n, 10)] = r.standard_normal(10)
    f[r.integers(0, n, 3)] = np.nan
    d = {"f": f, "i": np.arange(n)}
    t = td.table(d)
    try:
        keys = [("f", False, None)]
        return _bits(_run(td, t, keys)), _bits(oracle.sort(d, keys))
    finally:
        td.release(t)


def expr_keys(td, seed=12, n=ROWS):
    """Key expressions, evaluated over the input table: a*b DESC, then
    f + 1.0; the result holds the table's own columns."""
    r = np.random.default_rng(seed)
    d = {"a": r.integers(-50, 50, n), "b": r.integers(0, 10, n), "f": np.round(r.standard_normal(n), 1),
         "i": np.arange(n)}
    t = td.table(d)
    try:
        g = td.graph(t)
        try:
            k0 = g.op("mul", g.scan("a"), g.scan("b"))
            k1 = g.op("add", g.scan("f"), g.f64(1.0))
            res = g.execute(g.sort(g.const_table(t), [k0, k1], [1, 0]), optimize=False)
        finally:
            g.free()
        got = td.table_dict(res)
        td.release(res)
        full = dict(d, _k0=d["a"] * d["b"], _k1=d["f"] + 1.0)
        want = oracle.sort(full, [("_k0", True, None), ("_k1", False, None)])
        return _bits(got), _bits({k: want[k] for k in d})
    finally:
        td.release(t)


ALL = [i64_ties, f64_desc_nan_zero, f64_asc_nan_first, i32_key, two_keys, sym_key, head_of_sort, sort_of_group,
       small_int_keys, f64_zeros_two_keys, f64_zeros_small, expr_keys]


def same(got, want):
    assert list(got) == list(want), (list(got), list(want))
    for k in want:
        g, w = np.asarray(got[k]), np.asarray(want[k])
        assert len(g) == len(w), k
        assert np.array_equal(g.astype(w.dtype) if w.dtype != object else g, w), k
