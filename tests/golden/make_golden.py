"""Generate tests/golden/*.npz by running Teide itself (oracle/_ref/libteide_ref.so,
compiled from the reference's sources by oracle/Makefile) on small seeded
inputs of each workload shape.  Each fixture stores the inputs and Teide's
output, rows sorted by key (group-by) or by every column (join); the sort
fixture keeps Teide's row order, which is the thing under test.

    make -C oracle && python tests/golden/make_golden.py

The pipelines are the well-defined two-graph forms Teide runs correctly:
filter graph -> compacted table -> group graph (filter->group), and
join(filter(probe), build) -> group graph (filter->join->group).
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

from teide_b200 import workloads  # noqa: E402
from teide_b200.td import BOOL, I16, OP_AVG, OP_COUNT, OP_MAX, OP_MIN, OP_SUM, U8, Td  # noqa: E402
import oracle  # noqa: E402


def ref_filter_group(td, cols, pred, keys, aggs):
    """pred = (col, op, const); aggs = [(op, col)]."""
    t = td.table(cols)
    g = td.graph(t)
    c, op, k = pred
    kk = g.f64(k) if isinstance(k, float) else g.i64(k)
    t2 = g.execute(g.filter(g.const_table(t), g.op(op, g.scan(c), kk)), optimize=False)
    g.free()
    g = td.graph(t2)
    grp = g.group([g.scan(k) for k in keys], [a for a, _ in aggs], [g.scan(c) for _, c in aggs])
    r = g.execute(grp, optimize=False)
    g.free()
    out = td.table_dict(r)
    for x in (r, t2, t):
        td.release(x)
    return oracle.canonical(out, by=keys)


def ref_filter_join_group(td, build, probe, pred, lkey, rkey, keys, aggs, jt=0):
    b = td.table(build)
    p = td.table(probe)
    g = td.graph(p)
    c, op, k = pred
    j = g.join(g.filter(g.const_table(p), g.op(op, g.scan(c), g.i64(k))), [g.scan(lkey)],
               g.const_table(b), [g.scan(rkey)], jt)
    jr = g.execute(j, optimize=False)
    g.free()
    joined = td.table_dict(jr)
    g = td.graph(jr)
    grp = g.group([g.scan(k) for k in keys], [a for a, _ in aggs], [g.scan(c) for _, c in aggs])
    r = g.execute(grp, optimize=False)
    g.free()
    out = td.table_dict(r)
    for x in (r, jr, b, p):
        td.release(x)
    return oracle.canonical(out, by=keys), oracle.canonical(joined)


# sort fixtures: name -> (columns, Teide type tags, keys [(column, desc, nulls_first or -1)])
def sort_inputs():
    r = np.random.default_rng(105)
    n = 3000
    a = {"k": r.integers(0, 50, n), "i": np.arange(n), "v": r.standard_normal(n)}
    f = np.round(r.standard_normal(2000), 1)
    f[r.integers(0, 2000, 40)] = np.nan
    f[r.integers(0, 2000, 40)] = -0.0
    f[r.integers(0, 2000, 40)] = 0.0
    b = {"f": f, "i": np.arange(2000)}
    g = np.round(r.standard_normal(n), 0)
    g[r.integers(0, n, 600)] = -0.0
    g[r.integers(0, n, 600)] = 0.0
    c = {"f": g, "k": r.integers(0, 5, n), "i": np.arange(n)}
    d = {"b": r.integers(0, 2, n).astype(np.uint8), "h": r.integers(-300, 300, n).astype(np.int16),
         "u": r.integers(0, 256, n).astype(np.uint8), "i": np.arange(n)}
    return {
        "a": (a, {}, [("k", 0, -1)]),                                  # one I64 key, ties keep row order
        "b": (b, {}, [("f", 1, -1)]),                                  # F64 DESC: NaN first, -0.0 / +0.0 apart
        "c": (c, {}, [("f", 0, 1), ("k", 1, -1)]),                     # two keys: zeros equal, NaN-free
        "d": (d, {"b": BOOL, "h": I16, "u": U8}, [("b", 0, -1), ("h", 1, -1), ("u", 0, -1)]),
    }


def ref_sort(td, cols, tags, keys):
    t = td.table({k: ((v, tags[k]) if k in tags else v) for k, v in cols.items()})
    g = td.graph(t)
    nf = None if all(k[2] < 0 for k in keys) else [int(k[1] if k[2] < 0 else k[2]) for k in keys]
    r = g.execute(g.sort(g.const_table(t), [g.scan(k[0]) for k in keys], [int(k[1]) for k in keys], nf),
                  optimize=False)
    g.free()
    out = td.table_dict(r)
    td.release(r)
    td.release(t)
    return out


def save(name, **arrays):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **arrays)
    print(name, {k: v.shape for k, v in arrays.items()}, os.path.getsize(path), "bytes")


def main():
    td = Td(os.path.join(ROOT, "oracle", "_ref", "libteide_ref.so"))

    c1 = workloads.readme_table(n=20_000, seed=101)
    out = ref_filter_group(td, c1, ("flag", "eq", 0), ["region"], [(OP_SUM, "amount")])
    save("readme_small", **{"in_" + k: v for k, v in c1.items()}, **{"out_" + k: v for k, v in out.items()})

    c2 = workloads.zipf_group_table(n=30_000, seed=102, nkeys=1 << 12)
    aggs = [(OP_COUNT, "v1"), (OP_SUM, "v1"), (OP_MIN, "v1"), (OP_MAX, "v1"), (OP_AVG, "v2")]
    out = ref_filter_group(td, c2, ("v1", "gt", 0), ["key"], aggs)
    save("zipf_group_small", **{"in_" + k: v for k, v in c2.items()}, **{"out_" + k: v for k, v in out.items()})

    b3, p3 = workloads.join_tables(n_build=5_000, n_probe=30_000, seed=103)
    out, joined = ref_filter_join_group(td, b3, p3, ("qty", "gt", 10), "fk", "pk", ["cat"],
                                        [(OP_SUM, "price"), (OP_COUNT, "price")])
    save("join_group_small", **{"b_" + k: v for k, v in b3.items()}, **{"p_" + k: v for k, v in p3.items()},
         **{"out_" + k: v for k, v in out.items()}, **{"join_" + k: v for k, v in joined.items()})

    # outer joins with duplicates on both sides
    r = np.random.default_rng(104)
    left = {"id": r.integers(0, 300, 2_000).astype(np.int64), "val": r.integers(-50, 50, 2_000).astype(np.int64)}
    right = {"id": r.integers(100, 400, 1_500).astype(np.int64), "score": r.random(1_500)}
    res = {}
    for jt in (0, 1, 2):
        lt, rt = td.table(left), td.table(right)
        g = td.graph(lt)
        k = g.scan("id")
        jr = g.execute(g.join(g.const_table(lt), [k], g.const_table(rt), [k], jt), optimize=False)
        g.free()
        for nm, v in oracle.canonical(td.table_dict(jr)).items():
            res[f"j{jt}_{nm}"] = v
        for x in (jr, lt, rt):
            td.release(x)
    save("join_outer_small", **{"l_" + k: v for k, v in left.items()},
         **{"r_" + k: v for k, v in right.items()}, **res)

    arrays = {}
    for name, (cols, tags, keys) in sort_inputs().items():
        out = ref_sort(td, cols, tags, keys)
        arrays.update({f"{name}_in_{k}": v for k, v in cols.items()})
        arrays.update({f"{name}_out_{k}": v for k, v in out.items()})
        arrays[f"{name}_keys"] = np.array([f"{k}:{d}:{nf}" for k, d, nf in keys])
    save("sort_small", **arrays)


if __name__ == "__main__":
    main()
