"""Known-answer cases from Teide's own unit tests, written against the td.h API.

Each case builds the same tables and DAGs as the cited C test and asserts the
same answers.  They run on any library exporting td.h: on Teide itself
(tests/test_known_ref.py, CPU) -- which pins these translations -- and on
libteide_b200.so (tests/test_known_gpu.py, GPU).
"""
import numpy as np

from teide_b200.td import OP_AVG, OP_COUNT, OP_MAX, OP_MIN, OP_SUM, TdError

ID1 = np.array([1, 1, 2, 2, 3, 3, 1, 2, 3, 1], np.int64)
V1 = np.array([10, 20, 30, 40, 50, 60, 70, 80, 90, 100], np.int64)
V3 = np.array([1.5, 2.5, 3.5, 4.5, 5.5, 6.5, 7.5, 8.5, 9.5, 10.5])


def exec_table(td):
    """make_exec_table / make_test_table (test_exec.c:31-57, test_graph.c:33-58)."""
    return td.table({"id1": ID1, "v1": V1, "v3": V3})


def _run(td, tbl, build):
    g = td.graph(tbl)
    try:
        return g.execute(build(g), optimize=False)
    finally:
        g.free()


def case_comparisons(td):
    """test_exec.c:351-457 -- filter a vector, COUNT."""
    t = exec_table(td)
    want = {"eq": 1, "ne": 9, "lt": 4, "le": 5, "gt": 5}
    for op, n in want.items():
        r = _run(td, t, lambda g: g.op("count", g.filter(g.scan("v1"),
                                                         g.op(op, g.scan("v1"), g.i64(50)))))
        assert td.atom_value(r) == n, op
        td.release(r)
    r = _run(td, t, lambda g: g.op("count", g.filter(g.scan("v1"), g.op(
        "and", g.op("gt", g.scan("v1"), g.i64(20)), g.op("lt", g.scan("v1"), g.i64(80))))))
    assert td.atom_value(r) == 5
    td.release(r)
    r = _run(td, t, lambda g: g.op("count", g.filter(g.scan("v1"), g.op(
        "or", g.op("lt", g.scan("v1"), g.i64(20)), g.op("gt", g.scan("v1"), g.i64(90))))))
    assert td.atom_value(r) == 2
    td.release(r)
    td.release(t)


def case_filter_count(td):
    """test_graph.c:96-123 -- v1 >= 50 -> 6 rows."""
    t = exec_table(td)
    r = _run(td, t, lambda g: g.op("count", g.filter(g.scan("v1"),
                                                     g.op("ge", g.scan("v1"), g.i64(50)))))
    assert td.atom_value(r) == 6
    td.release(r)
    td.release(t)


def case_arithmetic_sum(td):
    """test_graph.c:128-150 -- SUM(v3 * 2.0) = 120."""
    t = exec_table(td)
    r = _run(td, t, lambda g: g.op("sum", g.op("mul", g.scan("v3"), g.f64(2.0))))
    assert abs(td.atom_value(r) - 120.0) < 1e-9
    td.release(r)
    td.release(t)


def _by_key(td, res, key_idx=0, val_idx=1):
    d = td.table_dict(res)
    cols = list(d.values())
    return dict(zip(cols[key_idx].tolist(), cols[val_idx].tolist())), d


def case_group_sum(td):
    """test_graph.c:154-200 -- group id1, SUM(v1) -> {1:200, 2:150, 3:200}."""
    t = exec_table(td)
    r = _run(td, t, lambda g: g.group([g.scan("id1")], [OP_SUM], [g.scan("v1")]))
    m, d = _by_key(td, r)
    assert m == {1: 200, 2: 150, 3: 200}
    assert list(d) == ["id1", "v1_sum"]
    td.release(r)
    td.release(t)


def case_group_affine(td):
    """test_graph.c:336-470 -- scalar and grouped aggregates of expressions."""
    t = exec_table(td)

    def scalar(ops, ins_fn):
        r = _run(td, t, lambda g: g.group([], ops, ins_fn(g)))
        d = td.table_dict(r)
        td.release(r)
        return [v[0] for v in d.values()]

    s, a = scalar([OP_SUM, OP_AVG], lambda g: [g.op("add", g.scan("v1"), g.i64(1))] * 2)
    assert s == 560 and abs(a - 56.0) < 1e-9
    s1, s2 = scalar([OP_SUM, OP_SUM], lambda g: [g.op("add", g.i64(1), g.scan("v1")),
                                                 g.op("sub", g.scan("v1"), g.i64(1))])
    assert (s1, s2) == (560, 540)
    (s,) = scalar([OP_SUM], lambda g: [g.op("add", g.scan("v1"), g.op("mul", g.i64(2), g.i64(1)))])
    assert s == 570
    s, a = scalar([OP_SUM, OP_AVG], lambda g: [
        g.op("mul", g.op("add", g.scan("v1"), g.i64(1)), g.i64(2)),
        g.op("add", g.op("add", g.scan("v1"), g.scan("id1")), g.i64(1))])
    assert s == 1120 and abs(a - 57.9) < 1e-9
    (s,) = scalar([OP_SUM], lambda g: [g.op("mul", g.i64(2), g.i64(1))])
    assert s == 20
    r = _run(td, t, lambda g: g.group([g.scan("id1")], [OP_SUM],
                                      [g.op("add", g.scan("v1"), g.i64(1))]))
    m, _ = _by_key(td, r)
    assert m == {1: 204, 2: 153, 3: 203}
    td.release(r)
    td.release(t)


def case_parallel_group_sum(td):
    """test_pool.c:131-216 -- 100K rows, id = i % 4, v = id + 1."""
    n = 100_000
    ids = np.arange(n, dtype=np.int64) % 4
    t = td.table({"id": ids, "v": ids + 1})
    r = _run(td, t, lambda g: g.group([g.scan("id")], [OP_SUM], [g.scan("v")]))
    m, _ = _by_key(td, r)
    assert m == {0: 25000, 1: 50000, 2: 75000, 3: 100000}
    td.release(r)
    td.release(t)


def case_parallel_min_max(td):
    """test_pool.c:218-270 -- MIN/MAX over F64 x = i - 50000."""
    n = 100_000
    t = td.table({"x": np.arange(n, dtype=np.float64) - 50000})
    r = _run(td, t, lambda g: g.op("min_op", g.scan("x")))
    assert td.atom_value(r) == -50000.0
    td.release(r)
    r = _run(td, t, lambda g: g.op("max_op", g.scan("x")))
    assert td.atom_value(r) == 49999.0
    td.release(r)
    td.release(t)


def _join(td, left, right, keys, jt):
    g = td.graph(left)
    try:
        ks = [g.scan(k) for k in keys]
        j = g.join(g.const_table(left), ks, g.const_table(right), ks, jt)
        return g.execute(j, optimize=False)
    finally:
        g.free()


def case_join_small(td):
    """test_exec.c:691-745 -- 3 x 4 rows, key 2 matches twice -> 4 rows."""
    left = td.table({"id": np.array([1, 2, 3]), "val": np.array([10, 20, 30])})
    right = td.table({"id": np.array([1, 2, 2, 3]), "score": np.array([100, 200, 201, 300])})
    r = _join(td, left, right, ["id"], 0)
    d = td.table_dict(r)
    assert len(d["id"]) == 4 and list(d) == ["id", "val", "score"]
    assert sorted(zip(d["id"], d["score"])) == [(1, 100), (2, 200), (2, 201), (3, 300)]
    for x in (r, left, right):
        td.release(x)


def case_join_large(td):
    """test_exec.c:747-832 -- 100K x 100K, each key twice per side -> 200K rows,
    SUM(score) = 99,999,000,000."""
    n = 100_000
    i = np.arange(n, dtype=np.int64)
    left = td.table({"id": i % 50000, "val": i})
    right = td.table({"id": i % 50000, "score": i * 10})
    r = _join(td, left, right, ["id"], 0)
    d = td.table_dict(r)
    assert len(d["score"]) == 200_000 and len(d) == 3
    assert int(d["score"].sum()) == 99_999_000_000
    for x in (r, left, right):
        td.release(x)


def case_join_asymmetric(td):
    """test_exec.c:834-915 -- 100 x 100K -> 100K rows, val = id * 7."""
    left = td.table({"id": np.arange(100, dtype=np.int64), "val": np.arange(100, dtype=np.int64) * 7})
    right = td.table({"id": np.arange(100_000, dtype=np.int64) % 100,
                      "score": np.arange(100_000, dtype=np.int64)})
    r = _join(td, left, right, ["id"], 0)
    d = td.table_dict(r)
    assert len(d["id"]) == 100_000
    assert np.array_equal(d["val"], d["id"] * 7)
    for x in (r, left, right):
        td.release(x)


def case_join_empty(td):
    """test_exec.c:917-1026 -- empty sides: 0 / 0 / 3 / 3 / 3 rows."""
    full = td.table({"id": np.array([1, 2, 3]), "val": np.array([10, 20, 30])})
    empty = td.table({"id": np.zeros(0, np.int64), "score": np.zeros(0, np.int64)})
    for l, rr, jt, n in ((full, empty, 0, 0), (empty, full, 0, 0), (full, empty, 1, 3),
                        (full, empty, 2, 3), (empty, full, 2, 3)):
        r = _join(td, l, rr, ["id"], jt)
        assert td.lib.td_table_nrows(r) == n, (jt, n)
        td.release(r)
    td.release(full)
    td.release(empty)


def case_join_left_large(td):
    """test_exec.c:1028-1099 -- LEFT join keeps all 100K left rows."""
    n = 100_000
    i = np.arange(n, dtype=np.int64)
    left = td.table({"id": i, "val": i * 10})
    right = td.table({"id": i * 2, "score": i * 100})
    r = _join(td, left, right, ["id"], 1)
    d = td.table_dict(r)
    assert len(d["id"]) == n
    m = d["id"] % 2 == 0
    assert np.array_equal(d["score"][m], d["id"][m] * 50)
    assert not d["score"][~m].any()
    for x in (r, left, right):
        td.release(x)


def case_join_full_large(td):
    """test_exec.c:1101-1152 -- FULL join of 0..79999 with 40000..119999 -> 120K."""
    i = np.arange(80_000, dtype=np.int64)
    left = td.table({"id": i})
    right = td.table({"id": i + 40000})
    r = _join(td, left, right, ["id"], 2)
    assert td.lib.td_table_nrows(r) == 120_000
    for x in (r, left, right):
        td.release(x)


def case_join_skewed(td):
    """test_exec.c:1154-1229 -- all left keys 42 -> 100K rows of score 294."""
    n = 100_000
    i = np.arange(n, dtype=np.int64)
    left = td.table({"id": np.full(n, 42, np.int64), "val": i})
    right = td.table({"id": i, "score": i * 7})
    r = _join(td, left, right, ["id"], 0)
    d = td.table_dict(r)
    assert len(d["score"]) == n and (d["score"] == 294).all()
    for x in (r, left, right):
        td.release(x)


def case_join_boundary(td):
    """test_exec.c:1231-1297 -- 65,537 x 65,537 identity join, each id once."""
    n = 65_537
    i = np.arange(n, dtype=np.int64)
    left = td.table({"id": i})
    right = td.table({"id": i})
    r = _join(td, left, right, ["id"], 0)
    d = td.table_dict(r)
    assert np.array_equal(np.sort(d["id"]), i)
    for x in (r, left, right):
        td.release(x)


def case_join_multikey(td):
    """test_exec.c:1299-1369 -- (I64, F64) keys -> 2 rows, scores {1000, 2000}."""
    left = td.table({"k1": np.array([1, 1, 2, 2, 3]), "k2": np.array([10.0, 20.0, 10.0, 20.0, 10.0]),
                     "val": np.array([100, 200, 300, 400, 500])})
    right = td.table({"k1": np.array([1, 2, 3]), "k2": np.array([10.0, 20.0, 30.0]),
                      "score": np.array([1000, 2000, 3000])})
    r = _join(td, left, right, ["k1", "k2"], 0)
    d = td.table_dict(r)
    assert sorted(d["score"].tolist()) == [1000, 2000]
    for x in (r, left, right):
        td.release(x)


def _sel_total(td, sel):
    """td_sel_meta(sel)->total_pass (td.h: the TD_SEL body starts with it)."""
    import ctypes as C
    typ, _, _ = td.header(sel)
    assert typ == 16, typ                             # TD_SEL
    return C.c_int64.from_address(sel + 32).value


def _sel_bits(td, sel, n):
    import ctypes as C
    n_segs = C.c_uint32.from_address(sel + 32 + 8).value
    off = 32 + 16 + ((n_segs + 7) & ~7) + 2 * ((n_segs + 3) & ~3)
    words = (n + 63) // 64
    return np.frombuffer(C.string_at(sel + off, 8 * words), np.uint64)


def case_sel_from_pred(td):
    """test_sel.c:42-64 -- BOOL [1,0,1,0,1] -> TD_SEL with total_pass 3."""
    b = td.vec(np.array([1, 0, 1, 0, 1], np.bool_))
    s = td.check(td.lib.td_sel_from_pred(b), "sel_from_pred")
    assert _sel_total(td, s) == 3
    assert int(_sel_bits(td, s, 5)[0]) == 0b10101
    td.release(s)
    td.release(b)


def case_sel_and(td):
    """test_sel.c:66-92 -- {1,1,0,0,1} AND {1,0,1,0,1} -> 2 passing."""
    a = td.vec(np.array([1, 1, 0, 0, 1], np.bool_))
    b = td.vec(np.array([1, 0, 1, 0, 1], np.bool_))
    sa = td.check(td.lib.td_sel_from_pred(a), "sel_from_pred")
    sb = td.check(td.lib.td_sel_from_pred(b), "sel_from_pred")
    s = td.check(td.lib.td_sel_and(sa, sb), "sel_and")
    assert _sel_total(td, s) == 2
    assert int(_sel_bits(td, s, 5)[0]) == 0b10001
    for x in (s, sa, sb, a, b):
        td.release(x)


def case_sel_large(td):
    """td_sel_from_pred over 5000 rows (five segments: NONE, ALL, MIX) --
    the bits and total match the BOOL vector (sel.c:128-161)."""
    import ctypes as C
    n = 5000
    m = np.zeros(n, np.bool_)
    m[1024:2048] = True
    m[2048:] = (np.arange(n - 2048) % 3) == 0
    b = td.vec(m)
    s = td.check(td.lib.td_sel_from_pred(b), "sel_from_pred")
    assert _sel_total(td, s) == int(m.sum())
    bits = _sel_bits(td, s, n)
    got = np.unpackbits(bits.view(np.uint8), bitorder="little")[:n].astype(bool)
    assert np.array_equal(got, m)
    flags = np.frombuffer(C.string_at(s + 48, 5), np.uint8)
    assert flags.tolist() == [0, 1, 2, 2, 2]
    td.release(s)
    td.release(b)


def case_sel_filter_integration(td):
    """test_sel.c:94-122 -- SUM(filter(x, x > 25)) over {10..50} = 120."""
    t = td.table({"x": np.array([10, 20, 30, 40, 50], np.int64)})
    r = _run(td, t, lambda g: g.op("sum", g.filter(g.scan("x"), g.op("gt", g.scan("x"), g.i64(25)))))
    assert td.atom_value(r) == 120
    td.release(r)
    td.release(t)


ALL = [case_comparisons, case_filter_count, case_arithmetic_sum, case_group_sum,
       case_group_affine, case_parallel_group_sum, case_parallel_min_max, case_join_small,
       case_join_large, case_join_asymmetric, case_join_empty, case_join_left_large,
       case_join_full_large, case_join_skewed, case_join_boundary, case_join_multikey,
       case_sel_from_pred, case_sel_and, case_sel_large, case_sel_filter_integration]
