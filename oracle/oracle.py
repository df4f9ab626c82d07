"""CPU oracle for the filter -> join -> group-by path.  TEST INFRASTRUCTURE ONLY.

A numpy restatement of what Teide's executor computes on this path (TeideDB/
teide, src/ops/exec.c), used by tests/, __graft_entry__.smoke() and the CPU
baseline leg of bench.py as the checker.  The product (teide_b200) never
imports it.

It is pinned two ways (tests/test_oracle.py):
  * against the known answers of Teide's own unit tests (test/test_exec.c,
    test_graph.c, test_pool.c, test_sel.c), and
  * against Teide itself: oracle/_ref/libteide_ref.so, compiled from the
    reference's sources by oracle/Makefile, runs the same DAGs, and the
    committed fixtures in tests/golden/ hold its outputs.

Semantics restated here, with the lines they follow:
  * comparisons: I64 vs I64 compare as integers, anything involving F64
    compares as double (expr_compile type promotion, exec.c:872-895);
  * selection = AND of the predicates of chained filters (td_sel_and,
    sel.c:167-189; exec.c:11717-11731);
  * group-by output: one row per distinct key tuple; key columns keep their
    type; SUM is I64 (wrapping) or F64, COUNT I64, AVG = sum / count as
    double, MIN/MAX keep the input type; names "<col>_sum", "_count",
    "_mean", "_min", "_max" (emit_agg_columns, exec.c:4632-4773).  Rows are
    returned in ascending key order (the direct-array order, exec.c:6330-6391);
    compare hash-method results after sorting by key;
  * join: every (left, right) pair with equal keys (join_keys_eq,
    exec.c:7754-7768); output = all left columns then right non-key columns
    (exec.c:8635-8655); LEFT keeps unmatched left rows, FULL also unmatched
    right rows, with the missing side zero-filled (gather_fn, exec.c:1910-1939);
  * sort: every key encoded as an order-preserving u64 (radix_encode_fn,
    exec.c:2739-2840) and the rows ordered stably by the keys, the first key
    most significant (radix_sort_run, exec.c:2647-2737 keeps equal keys in row
    order); SYM keys order by their strings (build_enum_rank, exec.c:2876-2975).
"""
from __future__ import annotations

import numpy as np

OP_SUM, OP_MIN, OP_MAX, OP_COUNT, OP_AVG = 50, 52, 53, 54, 55
SUFFIX = {OP_SUM: "_sum", OP_COUNT: "_count", OP_AVG: "_mean", OP_MIN: "_min", OP_MAX: "_max"}

CMP = {
    "eq": np.equal, "ne": np.not_equal, "lt": np.less,
    "le": np.less_equal, "gt": np.greater, "ge": np.greater_equal,
}


def compare(op: str, a, b) -> np.ndarray:
    """Element-wise comparison with Teide's promotion: int vs int stays
    integer, any float operand promotes both to double."""
    a = np.asarray(a)
    b = np.asarray(b)
    if a.dtype.kind == "f" or b.dtype.kind == "f":
        a = a.astype(np.float64)
        b = b.astype(np.float64)
    else:
        a = a.astype(np.int64)
        b = b.astype(np.int64)
    return CMP[op](a, b)


def conj(cols: dict, terms) -> np.ndarray:
    """AND of (column, op, constant) terms."""
    n = len(next(iter(cols.values())))
    m = np.ones(n, dtype=bool)
    for name, op, k in terms:
        m &= compare(op, cols[name], k)
    return m


def _key_ids(keys):
    """Dense ids of key tuples in ascending key order, plus the unique keys."""
    if len(keys) == 1:
        k = keys[0]
        if k.dtype.kind == "f":
            k = np.where(k == 0, 0.0, k)          # -0.0 groups with +0.0
        uniq, inv = np.unique(k, return_inverse=True)
        return inv.ravel(), [uniq]
    # lexicographic: first key most significant
    cols = [np.where(k == 0, 0.0, k) if k.dtype.kind == "f" else k for k in keys]
    order = np.lexsort(cols[::-1])
    sk = [c[order] for c in cols]
    if len(order):
        new = np.zeros(len(order), dtype=bool)
        new[0] = True
        for c in sk:
            new[1:] |= c[1:] != c[:-1]
        gid_sorted = np.cumsum(new) - 1
    else:
        new = np.zeros(0, dtype=bool)
        gid_sorted = np.zeros(0, dtype=np.int64)
    inv = np.empty(len(order), dtype=np.int64)
    inv[order] = gid_sorted
    uniq = [c[new] for c in sk]
    return inv, uniq


def group(keys: dict, aggs, mask=None) -> dict:
    """Group-by.  keys: {name: array}; aggs: [(op, name, array or None)].
    Returns {column name: array} in ascending key order."""
    names = list(keys)
    karr = [np.asarray(keys[k]) for k in names]
    n = len(karr[0]) if karr else (len(aggs[0][2]) if aggs and aggs[0][2] is not None else 0)
    if mask is None:
        mask = np.ones(n, dtype=bool)
    sel = np.nonzero(mask)[0]
    out = {}
    if karr:
        inv, uniq = _key_ids([k[sel] for k in karr])
        ng = len(uniq[0])
        for nm, u, k in zip(names, uniq, karr):
            out[nm] = u.astype(k.dtype)
    else:
        inv = np.zeros(len(sel), dtype=np.int64)
        ng = 1 if len(sel) else 0
    cnt = np.bincount(inv, minlength=ng).astype(np.int64)
    order = np.argsort(inv, kind="stable")
    starts = np.searchsorted(inv[order], np.arange(ng)) if ng else np.zeros(0, np.int64)
    for op, nm, arr in aggs:
        col = f"{nm}{SUFFIX[op]}"
        if op == OP_COUNT:
            out[col] = cnt
            continue
        v = np.asarray(arr)[sel][order]
        isf = v.dtype.kind == "f"
        if op in (OP_SUM, OP_AVG):
            if ng == 0:
                s = np.zeros(0, np.float64 if isf else np.int64)
            elif isf:
                s = np.add.reduceat(v.astype(np.float64), starts)
            else:
                with np.errstate(over="ignore"):
                    s = np.add.reduceat(v.astype(np.int64), starts)
            out[col] = s if op == OP_SUM else s.astype(np.float64) / cnt
        elif op == OP_MIN:
            out[col] = np.minimum.reduceat(v, starts) if ng else v[:0]
        elif op == OP_MAX:
            out[col] = np.maximum.reduceat(v, starts) if ng else v[:0]
    return out


def abs_bounds(keys: dict, aggs, mask=None) -> dict:
    """Per group, the scale of the F64 tolerance rule |got - want| <= 1e-12 *
    max(|want|, bound): sum |x| for an F64 SUM, sum |x| / count for AVG.
    Same arguments and row order as group(); only F64 SUM/AVG columns."""
    fa = [(op, nm, np.abs(np.asarray(a))) for op, nm, a in aggs
          if op in (OP_SUM, OP_AVG) and a is not None and np.asarray(a).dtype.kind == "f"]
    if not fa:
        return {}
    out = group(keys, fa, mask)
    for k in keys:                 # the key columns are not bounds
        out.pop(k, None)
    return out


def group_direct(key, aggs, mask=None, key_name="key") -> dict:
    """Group-by on one integer key through a direct array, slot = key - min
    (the DA path, exec.c:5948-6404; da_accum_row 5045-5099): the same result
    as group() for one integer key, in ascending key order, computed with
    scatter updates so that hundreds of millions of rows take seconds.
    Integer SUM wraps (np.add.at on int64, like exec.c:5075); F64 SUM adds
    in row order; AVG = sum / count; MIN/MAX keep the input type."""
    key = np.asarray(key)
    sel = None if mask is None else np.nonzero(mask)[0]
    k = key if sel is None else key[sel]
    out = {}
    if len(k) == 0:
        out[key_name] = key[:0].copy()
        for op, nm, arr in aggs:
            dt = np.int64 if op == OP_COUNT else (np.float64 if op == OP_AVG else
                                                  (np.float64 if np.asarray(arr).dtype.kind == "f" else np.int64))
            out[f"{nm}{SUFFIX[op]}"] = np.zeros(0, dt)
        return out
    lo = int(k.min())
    slot = (k.astype(np.int64) - lo)
    nslot = int(slot.max()) + 1
    cnt = np.bincount(slot, minlength=nslot).astype(np.int64)
    present = np.nonzero(cnt)[0]
    out[key_name] = (present + lo).astype(key.dtype)
    for op, nm, arr in aggs:
        col = f"{nm}{SUFFIX[op]}"
        if op == OP_COUNT:
            out[col] = cnt[present]
            continue
        v = np.asarray(arr)
        v = v if sel is None else v[sel]
        isf = v.dtype.kind == "f"
        if op in (OP_SUM, OP_AVG):
            if isf:
                acc = np.bincount(slot, weights=v.astype(np.float64), minlength=nslot)
            else:
                acc = np.zeros(nslot, np.int64)
                np.add.at(acc, slot, v.astype(np.int64))
            acc = acc[present]
            out[col] = acc if op == OP_SUM else acc.astype(np.float64) / cnt[present]
        elif op in (OP_MIN, OP_MAX):
            if isf:
                acc = np.full(nslot, np.inf if op == OP_MIN else -np.inf, v.dtype)
            else:
                info = np.iinfo(v.dtype)
                acc = np.full(nslot, info.max if op == OP_MIN else info.min, v.dtype)
            (np.minimum if op == OP_MIN else np.maximum).at(acc, slot, v)
            out[col] = acc[present]
    return out


def join_unique_direct(lkey, rkey, lmask=None):
    """(left row, right row) pairs of an inner equi-join on one integer key
    whose build-side (right) values are unique, through a direct map of the
    build keys: the pairs join_pairs() gives for that case (left-row order),
    at hundreds of millions of rows.  Raises if a build key repeats."""
    rkey = np.asarray(rkey).astype(np.int64)
    lkey = np.asarray(lkey).astype(np.int64)
    lsel = np.arange(len(lkey)) if lmask is None else np.nonzero(lmask)[0]
    if len(rkey) == 0 or len(lsel) == 0:
        return np.zeros(0, np.int64), np.zeros(0, np.int64)
    lo, hi = int(rkey.min()), int(rkey.max())
    row = np.full(hi - lo + 1, -1, np.int64)
    row[rkey - lo] = np.arange(len(rkey))
    if int((row >= 0).sum()) != len(rkey):
        raise ValueError("join_unique_direct: build keys repeat")
    lk = lkey[lsel]
    inr = (lk >= lo) & (lk <= hi)
    ri = np.full(len(lk), -1, np.int64)
    ri[inr] = row[lk[inr] - lo]
    hit = ri >= 0
    return lsel[hit].astype(np.int64), ri[hit]


def _join_ids(lkeys, rkeys):
    """Map key tuples of both sides onto shared dense ids."""
    nl = len(lkeys[0])
    both = [np.concatenate([np.asarray(a), np.asarray(b)]) for a, b in zip(lkeys, rkeys)]
    inv, _ = _key_ids(both)
    return inv[:nl], inv[nl:]


def join_pairs(lkeys, rkeys, join_type=0, lmask=None):
    """(left row, right row) pairs of an equi-join; -1 marks the missing side
    of an outer-join row.  Pairs come in left-row order, then right-row order
    within a left row, then unmatched right rows (full join)."""
    nl = len(lkeys[0])
    nr = len(rkeys[0])
    lsel = np.arange(nl) if lmask is None else np.nonzero(lmask)[0]
    if nr == 0 or len(lsel) == 0:
        li = lsel if join_type >= 1 else np.zeros(0, np.int64)
        ri = -np.ones(len(li), np.int64)
        if join_type == 2 and nr:
            li = np.concatenate([li, -np.ones(nr, np.int64)])
            ri = np.concatenate([ri, np.arange(nr)])
        return li.astype(np.int64), ri.astype(np.int64)
    lid, rid = _join_ids([np.asarray(k)[lsel] for k in lkeys], rkeys)
    nan_l = np.zeros(len(lsel), bool)
    nan_r = np.zeros(nr, bool)
    for a, b in zip(lkeys, rkeys):
        a = np.asarray(a)[lsel]
        if a.dtype.kind == "f":
            nan_l |= np.isnan(a)
        b = np.asarray(b)
        if b.dtype.kind == "f":
            nan_r |= np.isnan(b)
    rid = np.where(nan_r, -2, rid)
    ro = np.argsort(rid, kind="stable")
    rs = rid[ro]
    lo = np.searchsorted(rs, lid, "left")
    hi = np.searchsorted(rs, lid, "right")
    cnt = np.where(nan_l, 0, hi - lo)
    emit = np.where((cnt == 0) & (join_type >= 1), 1, cnt)
    li = np.repeat(lsel, emit)
    starts = np.repeat(lo, emit)
    within = np.arange(len(li)) - np.repeat(np.cumsum(emit) - emit, emit)
    matched = np.repeat(cnt > 0, emit)
    ri = np.where(matched, ro[np.minimum(starts + within, nr - 1)], -1)
    if join_type == 2:
        hit = np.zeros(nr, bool)
        hit[ri[ri >= 0]] = True
        un = np.nonzero(~hit)[0]
        li = np.concatenate([li, -np.ones(len(un), np.int64)])
        ri = np.concatenate([ri, un])
    return li.astype(np.int64), ri.astype(np.int64)


def gather(arr, idx):
    arr = np.asarray(arr)
    out = np.zeros(len(idx), arr.dtype)
    ok = idx >= 0
    out[ok] = arr[idx[ok]]
    return out


def join(left: dict, right: dict, lkey_names, rkey_names, join_type=0, lmask=None) -> dict:
    li, ri = join_pairs([left[k] for k in lkey_names], [right[k] for k in rkey_names],
                        join_type, lmask)
    out = {nm: gather(c, li) for nm, c in left.items()}
    for nm, c in right.items():
        if nm in rkey_names:
            continue
        out.setdefault(nm, gather(c, ri))
    return out


def canonical(d: dict, by=None) -> dict:
    """Rows sorted by the given columns (default: all, in column order)."""
    cols = list(d) if by is None else list(by)
    if not cols or len(d[cols[0]]) == 0:
        return {k: np.asarray(v) for k, v in d.items()}
    keys = []
    for c in cols:
        v = np.asarray(d[c])
        keys.append(v.view(np.int64) if v.dtype == np.float64 else v)
    order = np.lexsort(keys[::-1])
    return {k: np.asarray(v)[order] for k, v in d.items()}


def sort_code(values, desc=False, nulls_first=None, kind=None, zero_eq=False):
    """The u64 code radix_encode_fn (exec.c:2739-2840) gives each value:
    integers flip the sign bit (I32 / DATE / TIME at 32 bits, I16 at 16),
    BOOL / U8 keep their unsigned byte (sort_cmp, exec.c:2538-2547), F64 maps
    to IEEE order (-0.0 before +0.0, or equal to it with zero_eq, as in
    sort_cmp) with NaN smallest or largest by nulls_first (default: DESC),
    strings (SYM) to the rank of their bytes among the distinct strings, and
    DESC complements the code."""
    nf = desc if nulls_first is None else nulls_first
    v = np.asarray(values)
    if kind == "sym" or v.dtype.kind in ("O", "U", "S"):
        b = [x.encode() if isinstance(x, str) else bytes(x) for x in v]
        uniq = sorted(set(b))
        rank = {x: i for i, x in enumerate(uniq)}
        e = np.array([rank[x] for x in b], dtype=np.uint64)
    elif v.dtype == np.bool_ or v.dtype == np.uint8:
        e = v.astype(np.uint64)
    elif v.dtype == np.int16:
        e = (v.view(np.uint16) ^ np.uint16(0x8000)).astype(np.uint64)
    elif v.dtype == np.float64:
        if zero_eq:
            v = np.where(v == 0.0, 0.0, v)   # -0.0 -> +0.0; NaN and the rest unchanged
        bits = v.view(np.uint64)
        mask = (np.uint64(0) - (bits >> np.uint64(63))) | np.uint64(1 << 63)
        e = bits ^ mask
        nan_e = np.uint64(0) if (bool(nf) ^ bool(desc)) else np.uint64(0xFFFFFFFFFFFFFFFF)
        e = np.where(np.isnan(v), (~nan_e) if desc else nan_e, e).astype(np.uint64)
        return e if not desc else np.where(np.isnan(v), e, ~e)
    elif v.dtype.itemsize == 4:
        e = (v.astype(np.int32).view(np.uint32) ^ np.uint32(1 << 31)).astype(np.uint64)
    else:
        e = v.astype(np.int64).view(np.uint64) ^ np.uint64(1 << 63)
    return ~e if desc else e


def sort(cols: dict, keys, limit=None) -> dict:
    """Rows of `cols` ordered by keys [(name, desc, nulls_first)] (stable,
    first key most significant), cut to the first `limit` rows when given.
    A SYM key column is passed as its strings.  Teide radix-sorts (exec.c:
    3426-3453) one key of a radix type over more than 64 rows; otherwise its
    comparator decides, where -0.0 equals +0.0 (zero_eq)."""
    n = len(next(iter(cols.values()))) if cols else 0
    small = {np.dtype(np.bool_), np.dtype(np.uint8), np.dtype(np.int16)}
    zero_eq = n <= 64 or len(keys) > 1 or any(np.asarray(cols[k[0]]).dtype in small for k in keys)
    codes = [sort_code(cols[name], desc, nf, zero_eq=zero_eq) for name, desc, nf in keys]
    order = np.lexsort(codes[::-1]) if codes else np.arange(n)
    if limit is not None:
        order = order[:limit]
    return {k: np.asarray(v)[order] for k, v in cols.items()}
