"""DAG builders for the filter -> (join ->) group pipelines, shared by the GPU
parity tests, the smoke test and the benchmark.  Each runs through the
td.h API (td_execute) of whatever library the Td binding wraps."""
import numpy as np

from teide_b200.td import OP_COUNT


def const(g, k):
    return g.f64(k) if isinstance(k, float) else g.i64(k)


def _result(td, r, as_dict):
    """The result as {name: numpy array}, or just released (as_dict False:
    the query's host td_t result is produced and dropped unread)."""
    out = td.table_dict(r) if as_dict else None
    td.release(r)
    return out


def readme_group(td, tbl, pred, keys, aggs, as_dict=True):
    """One graph: group keys and aggregate inputs are td_filter(scan, pred)
    vectors sharing one predicate (README.md's filter + group + sum)."""
    g = td.graph(tbl)
    try:
        c, op, k = pred
        p = g.op(op, g.scan(c), const(g, k))
        ks = [g.filter(g.scan(name), p) for name in keys]
        ins = [g.filter(g.scan(name), p) for _, name in aggs]
        r = g.execute(g.group(ks, [a for a, _ in aggs], ins), optimize=True)
    finally:
        g.free()
    return _result(td, r, as_dict)


def two_graph_group(td, tbl, pred, keys, aggs, as_dict=True):
    """Filter graph -> compacted table -> group graph."""
    g = td.graph(tbl)
    try:
        c, op, k = pred
        t2 = g.execute(g.filter(g.const_table(tbl), g.op(op, g.scan(c), const(g, k))))
    finally:
        g.free()
    g = td.graph(t2)
    try:
        r = g.execute(g.group([g.scan(n) for n in keys], [a for a, _ in aggs],
                              [g.scan(n) for _, n in aggs]))
    finally:
        g.free()
    out = _result(td, r, as_dict)
    td.release(t2)
    return out


def fused_join_group(td, build_t, probe_t, pred, lkey, rkey, keys, aggs, join_type=0, as_dict=True):
    """One graph bound to no table: group over join(filter(probe), build)."""
    g = td.graph(None)
    try:
        c, op, k = pred
        left = g.filter(g.const_table(probe_t), g.op(op, g.scan(c), const(g, k)))
        g.join(left, [g.scan(lkey)], g.const_table(build_t), [g.scan(rkey)], join_type)
        grp = g.group([g.scan(n) for n in keys], [a for a, _ in aggs], [g.scan(n) for _, n in aggs])
        r = g.execute(grp)
    finally:
        g.free()
    return _result(td, r, as_dict)


def join_then_group(td, build_t, probe_t, pred, lkey, rkey, keys, aggs, join_type=0, as_dict=True):
    """Two calls: materialized join, then a group graph over its result.
    Returns (groups, joined rows) as {name: numpy array}; with as_dict False
    both host results are produced and dropped unread, so a timed step holds
    only the engine's own work."""
    g = td.graph(probe_t)
    try:
        c, op, k = pred
        left = g.filter(g.const_table(probe_t), g.op(op, g.scan(c), const(g, k)))
        jr = g.execute(g.join(left, [g.scan(lkey)], g.const_table(build_t), [g.scan(rkey)], join_type))
    finally:
        g.free()
    joined = td.table_dict(jr) if as_dict else None
    g = td.graph(jr)
    try:
        r = g.execute(g.group([g.scan(n) for n in keys], [a for a, _ in aggs],
                              [g.scan(n) for _, n in aggs]))
    finally:
        g.free()
    out = _result(td, r, as_dict)
    td.release(jr)
    return out, joined


def f64_tolerance_ok(got, want, abs_sum, rel=1e-12):
    """|got - want| <= rel * max(|want|, sum |x|) elementwise."""
    scale = np.maximum(np.abs(want), abs_sum)
    return bool(np.all(np.abs(got - want) <= rel * np.maximum(scale, 1e-300)))


CONFIG3_AGGS = [(None, "price"), (OP_COUNT, "price")]


def group_sorted(td, tbl, pred, keys, aggs, sort_col, desc=True, as_dict=True):
    """One graph: README-form filter + group-by, its result sorted by
    sort_col (td_sort_op over the group node)."""
    g = td.graph(tbl)
    try:
        c, op, k = pred
        p = g.op(op, g.scan(c), const(g, k))
        ks = [g.filter(g.scan(name), p) for name in keys]
        ins = [g.filter(g.scan(name), p) for _, name in aggs]
        grp = g.group(ks, [a for a, _ in aggs], ins)
        r = g.execute(g.sort(grp, [g.scan(sort_col)], [int(desc)]), optimize=True)
    finally:
        g.free()
    return _result(td, r, as_dict)


def two_graph_group_sorted(td, tbl, pred, keys, aggs, sort_col, desc=True):
    """Filter graph -> compacted table -> group graph -> sort graph."""
    g = td.graph(tbl)
    try:
        c, op, k = pred
        t2 = g.execute(g.filter(g.const_table(tbl), g.op(op, g.scan(c), const(g, k))))
    finally:
        g.free()
    g = td.graph(t2)
    try:
        grp = g.execute(g.group([g.scan(n) for n in keys], [a for a, _ in aggs], [g.scan(n) for _, n in aggs]))
    finally:
        g.free()
    g = td.graph(grp)
    try:
        r = g.execute(g.sort(g.const_table(grp), [g.scan(sort_col)], [int(desc)]), optimize=False)
    finally:
        g.free()
    td.release(grp)
    td.release(t2)
    td.release(r)


class Prepared:
    """A query DAG built (and passed through td_optimize) once and executed
    any number of times, like a prepared statement: each run() is one
    td_execute of the same graph, whose result is produced and then either
    returned as {name: numpy array} (as_dict) or released unread."""

    def __init__(self, td, tbl, build, optimize=True):
        self.td = td
        self.g = td.graph(tbl)
        try:
            root = build(self.g)
            if optimize:
                root = td.lib.td_optimize(self.g.g, root) or root
        except Exception:
            self.g.free()
            raise
        self.root = root

    def run(self, as_dict=False):
        r = self.td.check(self.td.lib.td_execute(self.g.g, self.root), "execute")
        return _result(self.td, r, as_dict)

    def free(self):
        self.g.free()


def prepared_readme_group(td, tbl, pred, keys, aggs):
    """readme_group's DAG, prepared."""
    def build(g):
        c, op, k = pred
        p = g.op(op, g.scan(c), const(g, k))
        return g.group([g.filter(g.scan(n), p) for n in keys], [a for a, _ in aggs],
                       [g.filter(g.scan(n), p) for _, n in aggs])
    return Prepared(td, tbl, build)


def prepared_fused_join_group(td, build_t, probe_t, pred, lkey, rkey, keys, aggs, join_type=0):
    """fused_join_group's DAG, prepared."""
    def build(g):
        c, op, k = pred
        left = g.filter(g.const_table(probe_t), g.op(op, g.scan(c), const(g, k)))
        g.join(left, [g.scan(lkey)], g.const_table(build_t), [g.scan(rkey)], join_type)
        return g.group([g.scan(n) for n in keys], [a for a, _ in aggs], [g.scan(n) for _, n in aggs])
    return Prepared(td, None, build)


def prepared_group_sorted(td, tbl, pred, keys, aggs, sort_col, desc=True):
    """group_sorted's DAG, prepared."""
    def build(g):
        c, op, k = pred
        p = g.op(op, g.scan(c), const(g, k))
        grp = g.group([g.filter(g.scan(n), p) for n in keys], [a for a, _ in aggs],
                      [g.filter(g.scan(n), p) for _, n in aggs])
        return g.sort(grp, [g.scan(sort_col)], [int(desc)])
    return Prepared(td, tbl, build)
