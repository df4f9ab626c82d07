"""Row-sharded filter -> (join ->) group-by over several GPUs.

One process per GPU (torch.distributed; NCCL on GPUs, gloo on CPU).  Every
rank holds a contiguous shard of the rows (and, for a join, the whole build
side) and runs the fused query on its own GPU through td_execute.  The only
exchange is the merge of partial group results:

  partial aggregates  SUM -> SUM, COUNT -> COUNT, MIN -> MIN, MAX -> MAX,
                      AVG -> SUM + COUNT (divided after the merge), so every
                      partial merges by sum / min / max;
  few groups          ("gather") every rank all-gathers all partial rows and
                      merges them, so each ends with the whole result;
  many groups         ("alltoall") each partial row goes to the rank that owns
                      its key (a hash of the key columns), one all-to-all moves
                      them, and each owner merges its share; the owners' parts
                      are disjoint and together are the result.

Partial results never leave the GPUs: each rank's local query runs with
td_execute_device, so its partial groups stay in device memory and cross only
NVLink (NCCL), and the merge of the gathered rows is itself a group-by run by
this library on the device (merge_device: tdg_group_run over the rows).  Only
the merged result is copied to the host.  Merged output is in ascending key
order (lexicographic over the key columns), like the direct-array emit of a
single GPU.  The local executor and the merge are parameters so the exchange
can be exercised on CPU ranks (gloo) with partial results and a merge from
the test's oracle; the product path passes the td_execute_device and
tdg_group_run ones.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch
import torch.distributed as dist

from .td import OP_AVG, OP_COUNT, OP_MAX, OP_MIN, OP_SUM

SUFFIX = {OP_SUM: "_sum", OP_COUNT: "_count", OP_AVG: "_mean", OP_MIN: "_min", OP_MAX: "_max"}


def partial_plan(aggs):
    """aggs [(op, col)] -> (partial aggs, finalize steps).  A finalize step is
    ("id", i) or ("avg", i_sum, i_count) over partial indices."""
    parts, steps = [], []

    def add(op, col):
        if (op, col) not in parts:
            parts.append((op, col))
        return parts.index((op, col))

    for op, col in aggs:
        if op == OP_AVG:
            steps.append(("avg", add(OP_SUM, col), add(OP_COUNT, col)))
        else:
            steps.append(("id", add(op, col)))
    return parts, steps


def _key_hash(keys: torch.Tensor) -> torch.Tensor:
    """A mixing hash of int64 key rows (n, nk) -> int64 (n,), non-negative."""
    h = torch.zeros(keys.shape[0], dtype=torch.int64, device=keys.device)
    for j in range(keys.shape[1]):
        x = keys[:, j] ^ (h * 31 + 0x9E3779B9)
        x = (x ^ (x >> 31)) * 0x7FB5D329728EA185
        h = x ^ (x >> 27)
    return h & 0x7FFFFFFFFFFFFFFF


_I64, _F64 = 6, 7


def merge_device(td, keys: torch.Tensor, vals: list, ops: list):
    """The merge of gathered partial rows is itself a group-by: keys (n, nk)
    int64 on the GPU, vals[i] (n,) int64 or float64, merged by ops[i] --
    SUM of the partial SUMs and COUNTs, MIN of the MINs, MAX of the MAXs --
    through the library's own group-by (tdg_group_run) on the device, with
    the key ranges of the rows so the planner can take a direct array.
    Returns (unique keys (g, nk), merged vals) on the device, ascending by
    key (the direct array's order; a hash-method result is sorted after)."""
    from . import device_abi
    from .tdg import GroupDesc, GroupOut, GroupPlan, col
    T = device_abi()
    n, nk = keys.shape
    if n == 0:
        return keys, [v[:0] for v in vals]
    kcols = [keys[:, j].contiguous() for j in range(nk)]
    if nk == 0:                                   # no group keys: one group
        kcols = [torch.zeros(n, dtype=torch.int64, device=keys.device)]
    vals = [v.contiguous() for v in vals]
    d = GroupDesc()
    d.nrows = n
    d.n_keys = len(kcols)
    d.n_aggs = len(vals)
    for j, k in enumerate(kcols):
        d.keys[j] = col(k.data_ptr(), _I64)
        lo, hi = torch.aminmax(k)
        d.key_min[j], d.key_max[j] = int(lo), int(hi)
    d.have_range = 1
    for a, (v, op) in enumerate(zip(vals, ops)):
        d.aggs[a].op = OP_SUM if op == OP_COUNT else op
        d.aggs[a].in_ = col(v.data_ptr(), _F64 if v.dtype == torch.float64 else _I64)
    plan = GroupPlan()
    st = T.tdg_group_plan_make(C.byref(d), 0, C.byref(plan))
    if st:
        raise RuntimeError(f"tdg_group_plan_make: {st}")
    ws = torch.empty(max(int(plan.ws_bytes), 1), dtype=torch.uint8, device=keys.device)
    o = GroupOut()
    ok = [torch.empty(max(plan.max_groups, 1), dtype=torch.int64, device=keys.device) for _ in kcols]
    ov = [torch.empty(max(plan.max_groups, 1), dtype=v.dtype, device=keys.device) for v in vals]
    for j, b in enumerate(ok):
        o.keys[j] = b.data_ptr()
    for a, b in enumerate(ov):
        o.aggs[a] = b.data_ptr()
    ng = torch.zeros(1, dtype=torch.int64, device=keys.device)
    o.d_n_groups = ng.data_ptr()
    st = T.tdg_group_run(C.byref(d), None, None, C.byref(plan), ws.data_ptr(), C.byref(o),
                         torch.cuda.current_stream(keys.device).cuda_stream)
    if st:
        raise RuntimeError(f"tdg_group_run: {st}")
    g = int(ng.item())
    uk = torch.stack([b[:g] for b in ok], 1) if nk else torch.zeros((g, 0), dtype=torch.int64, device=keys.device)
    mv = [b[:g] for b in ov]
    if plan.method != 1 and nk:                   # hash method: table order -> ascending keys
        order = torch.arange(g, device=keys.device)
        for j in reversed(range(nk)):
            order = order[torch.argsort(uk[order, j], stable=True)]
        uk, mv = uk[order], [m[order] for m in mv]
    return uk, mv


def _all_gather_rows(t: torch.Tensor, group=None) -> torch.Tensor:
    """Concatenate a (n_r, ...) tensor of every rank (n_r may differ)."""
    world = dist.get_world_size(group)
    n = torch.tensor([t.shape[0]], dtype=torch.int64, device=t.device)
    ns = [torch.zeros_like(n) for _ in range(world)]
    dist.all_gather(ns, n, group=group)
    ns = [int(x.item()) for x in ns]
    m = max(ns) if ns else 0
    pad = torch.zeros((m,) + tuple(t.shape[1:]), dtype=t.dtype, device=t.device)
    pad[:t.shape[0]] = t
    bufs = [torch.empty_like(pad) for _ in range(world)]
    dist.all_gather(bufs, pad, group=group)
    return torch.cat([b[:k] for b, k in zip(bufs, ns)], 0)


def _all_to_all_rows(t: torch.Tensor, dest: torch.Tensor, group=None) -> torch.Tensor:
    """Send row i of t to rank dest[i]; returns the rows this rank received."""
    world = dist.get_world_size(group)
    order = torch.argsort(dest, stable=True)
    t = t[order]
    send = torch.bincount(dest, minlength=world).to(torch.int64)
    recv = torch.empty_like(send)
    dist.all_to_all_single(recv, send, group=group)
    out = torch.empty((int(recv.sum().item()),) + tuple(t.shape[1:]), dtype=t.dtype, device=t.device)
    dist.all_to_all_single(out, t.contiguous(), [int(x) for x in recv.tolist()],
                           [int(x) for x in send.tolist()], group=group)
    return out


def exchange_and_merge(part: dict, key_names, parts, steps, strategy="auto", group=None,
                       device="cuda", gather_limit=1 << 20, merge=None, td=None):
    """Merge this rank's partial result `part` ({name: tensor on `device`, or
    numpy}) with every other rank's.  Returns {name: numpy} with the final
    columns: the whole result ("gather"), or this rank's disjoint share
    ("alltoall").  `merge(keys, vals, ops)` combines rows of equal keys; by
    default the library's group-by on the GPU (merge_device)."""
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    pnames = [f"{c}{SUFFIX[op]}" for op, c in parts]

    def t(x):
        return x if isinstance(x, torch.Tensor) else torch.as_tensor(np.ascontiguousarray(x), device=device)
    keys = torch.stack([t(part[k]).to(torch.int64) for k in key_names], 1) if key_names else \
        torch.zeros((len(part[pnames[0]]), 0), dtype=torch.int64, device=device)
    vals = [t(part[n]) for n in pnames]
    ops = [op for op, _ in parts]
    if world > 1:
        if strategy == "auto":
            n = torch.tensor([keys.shape[0]], dtype=torch.int64, device=device)
            dist.all_reduce(n, op=dist.ReduceOp.MAX, group=group)
            strategy = "gather" if int(n.item()) * world <= gather_limit else "alltoall"
        # one matrix of 8-byte words per row: keys, then the values' bits
        words = torch.cat([keys] + [v.view(torch.int64).reshape(-1, 1) if v.dtype == torch.float64
                                    else v.to(torch.int64).reshape(-1, 1) for v in vals], 1) \
            if vals else keys
        if strategy == "gather":
            words = _all_gather_rows(words, group)
        else:
            dest = (_key_hash(keys) % world) if keys.shape[1] else torch.zeros(keys.shape[0], dtype=torch.int64,
                                                                               device=device)
            words = _all_to_all_rows(words, dest, group)
        nk = keys.shape[1]
        keys = words[:, :nk]
        vals = [words[:, nk + i].contiguous().view(torch.float64) if v.dtype == torch.float64
                else words[:, nk + i].to(v.dtype) for i, v in enumerate(vals)]
    if merge is None:
        uk, mv = merge_device(td, keys, vals, ops)
    else:
        uk, mv = merge(keys, vals, ops)
    out = {k: uk[:, j].cpu().numpy() for j, k in enumerate(key_names)}
    for s in steps:
        if s[0] == "id":
            op, col_ = parts[s[1]]
            out[f"{col_}{SUFFIX[op]}"] = mv[s[1]].cpu().numpy()
        else:
            col_ = parts[s[1]][1]
            out[f"{col_}_mean"] = (mv[s[1]].to(torch.float64) / mv[s[2]].to(torch.float64)).cpu().numpy()
    return out


# ---- the td_execute local executors ------------------------------------------------

class _DevCol:
    """A device buffer seen through __cuda_array_interface__ (no copy)."""

    def __init__(self, ptr, n, typestr):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": typestr, "data": (ptr, False),
                                         "version": 3, "strides": None}


def _device_part(td, r):
    """{name: tensor} viewing the device columns of a td_execute_device
    result r (kept alive in the dict under "_result"; release it after use)."""
    L = td.lib
    L.td_gpu_col_data.restype = C.c_void_p
    L.td_gpu_col_data.argtypes = [C.c_void_p]
    out = {"_result": r}
    for j in range(L.td_table_ncols(r)):
        c = L.td_table_get_col_idx(r, j)
        typ, _, n = td.header(c)
        ptr = L.td_gpu_col_data(c)
        name = td.sym_name(L.td_table_col_name(r, j))
        if typ not in (_I64, _F64):
            raise NotImplementedError("sharded partials: only 8-byte integer and F64 result columns")
        if not ptr or n == 0:
            out[name] = torch.zeros(0, dtype=torch.float64 if typ == _F64 else torch.int64, device="cuda")
            continue
        out[name] = torch.as_tensor(_DevCol(ptr, n, "<f8" if typ == _F64 else "<i8"), device="cuda")
    return out


def _execute_device(td, g, root):
    L = td.lib
    L.td_execute_device.restype = C.c_void_p
    L.td_execute_device.argtypes = [C.c_void_p, C.c_void_p]
    return _device_part(td, td.check(L.td_execute_device(g.g, root), "td_execute_device"))


def local_group(td, tbl, pred, keys, parts):
    """Partial group-by of this rank's shard, left on its GPU: README form
    when pred is given (pred = (column, op, constant)), else a plain group
    graph."""
    from .serve import _const
    g = td.graph(tbl)
    try:
        if pred:
            c, op, k = pred
            p = g.op(op, g.scan(c), _const(g, k))
            ks = [g.filter(g.scan(n), p) for n in keys]
            ins = [g.filter(g.scan(n), p) for _, n in parts]
        else:
            ks = [g.scan(n) for n in keys]
            ins = [g.scan(n) for _, n in parts]
        return _execute_device(td, g, g.group(ks, [a for a, _ in parts], ins))
    finally:
        g.free()


def local_join_group(td, build_t, probe_t, pred, lkey, rkey, keys, parts):
    """Partial group-by over join(filter(probe shard), build), one fused
    graph, left on this rank's GPU."""
    from .serve import _const
    g = td.graph(None)
    try:
        c, op, k = pred
        left = g.filter(g.const_table(probe_t), g.op(op, g.scan(c), _const(g, k)))
        g.join(left, [g.scan(lkey)], g.const_table(build_t), [g.scan(rkey)], 0)
        return _execute_device(td, g, g.group([g.scan(n) for n in keys], [a for a, _ in parts],
                                              [g.scan(n) for _, n in parts]))
    finally:
        g.free()


def _finish(td, part, run):
    try:
        return run()
    finally:
        r = part.pop("_result", None) if isinstance(part, dict) else None
        if r and td is not None:
            td.release(r)


def sharded_group(td, tbl, keys, aggs, pred=None, strategy="auto", group=None, device="cuda", local=None,
                  merge=None):
    """Filter + group-by of the union of every rank's `tbl` shard."""
    parts, steps = partial_plan(aggs)
    part = (local or local_group)(td, tbl, pred, keys, parts)
    return _finish(td, part, lambda: exchange_and_merge(part, keys, parts, steps, strategy, group, device,
                                                        merge=merge, td=td))


def sharded_join_group(td, build_t, probe_t, pred, lkey, rkey, keys, aggs, strategy="auto", group=None,
                       device="cuda", local=None, merge=None):
    """Filter + join + group-by: probe rows sharded, build side on every rank."""
    parts, steps = partial_plan(aggs)
    part = (local or local_join_group)(td, build_t, probe_t, pred, lkey, rkey, keys, parts)
    return _finish(td, part, lambda: exchange_and_merge(part, keys, parts, steps, strategy, group, device,
                                                        merge=merge, td=td))
