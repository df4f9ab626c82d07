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

Merged output is in ascending key order (lexicographic over the key
columns), like the direct-array emit of a single GPU.  The local executor is
a parameter so the exchange and merge can be exercised on CPU ranks with any
partial-result provider; the product path passes the td_execute one.
"""
from __future__ import annotations

import numpy as np
import torch
import torch.distributed as dist

from .td import OP_AVG, OP_COUNT, OP_MAX, OP_MIN, OP_SUM

SUFFIX = {OP_SUM: "_sum", OP_COUNT: "_count", OP_AVG: "_mean", OP_MIN: "_min", OP_MAX: "_max"}
_REDUCE = {OP_SUM: "sum", OP_COUNT: "sum", OP_MIN: "amin", OP_MAX: "amax"}


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


def merge(keys: torch.Tensor, vals: list, ops: list):
    """Rows of partial results (keys (n, nk) int64, vals[i] (n,)) -> one row
    per distinct key in ascending order, vals merged by ops[i]."""
    if keys.shape[0] == 0:
        return keys, [v[:0] for v in vals]
    if keys.shape[1] == 0:                      # no group keys: one group
        uk = keys[:1]
        inv = torch.zeros(keys.shape[0], dtype=torch.int64, device=keys.device)
    else:
        uk, inv = torch.unique(keys, dim=0, sorted=True, return_inverse=True)
    out = []
    for v, op in zip(vals, ops):
        r = torch.zeros(uk.shape[0], dtype=v.dtype, device=v.device)
        out.append(r.scatter_reduce_(0, inv, v, reduce=_REDUCE[op], include_self=False))
    return uk, out


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
                       device="cpu", gather_limit=1 << 20):
    """Merge this rank's partial result `part` ({name: numpy}) with every
    other rank's.  Returns {name: numpy} with the final columns: the whole
    result ("gather"), or this rank's disjoint share ("alltoall")."""
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    pnames = [f"{c}{SUFFIX[op]}" for op, c in parts]
    keys = torch.stack([torch.as_tensor(np.ascontiguousarray(part[k]), device=device).to(torch.int64)
                        for k in key_names], 1) if key_names else \
        torch.zeros((len(part[pnames[0]]), 0), dtype=torch.int64, device=device)
    vals = [torch.as_tensor(np.ascontiguousarray(part[n]), device=device) for n in pnames]
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
    uk, mv = merge(keys, vals, ops)
    out = {k: uk[:, j].cpu().numpy() for j, k in enumerate(key_names)}
    for s in steps:
        if s[0] == "id":
            op, col = parts[s[1]]
            out[f"{col}{SUFFIX[op]}"] = mv[s[1]].cpu().numpy()
        else:
            col = parts[s[1]][1]
            out[f"{col}_mean"] = (mv[s[1]].to(torch.float64) / mv[s[2]].to(torch.float64)).cpu().numpy()
    return out


# ---- the td_execute local executors ------------------------------------------------

def local_group(td, tbl, pred, keys, parts):
    """Partial group-by of this rank's shard: README form when pred is given
    (pred = (column, op, constant)), else a plain group graph."""
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
        r = td.check(td.lib.td_execute(g.g, g.group(ks, [a for a, _ in parts], ins)), "td_execute")
    finally:
        g.free()
    out = td.table_dict(r)
    td.release(r)
    return out


def local_join_group(td, build_t, probe_t, pred, lkey, rkey, keys, parts):
    """Partial group-by over join(filter(probe shard), build), one fused graph."""
    from .serve import _const
    g = td.graph(None)
    try:
        c, op, k = pred
        left = g.filter(g.const_table(probe_t), g.op(op, g.scan(c), _const(g, k)))
        g.join(left, [g.scan(lkey)], g.const_table(build_t), [g.scan(rkey)], 0)
        root = g.group([g.scan(n) for n in keys], [a for a, _ in parts], [g.scan(n) for _, n in parts])
        r = td.check(td.lib.td_execute(g.g, root), "td_execute")
    finally:
        g.free()
    out = td.table_dict(r)
    td.release(r)
    return out


def sharded_group(td, tbl, keys, aggs, pred=None, strategy="auto", group=None, device="cuda", local=None):
    """Filter + group-by of the union of every rank's `tbl` shard."""
    parts, steps = partial_plan(aggs)
    part = (local or local_group)(td, tbl, pred, keys, parts)
    return exchange_and_merge(part, keys, parts, steps, strategy, group, device)


def sharded_join_group(td, build_t, probe_t, pred, lkey, rkey, keys, aggs, strategy="auto", group=None,
                       device="cuda", local=None):
    """Filter + join + group-by: probe rows sharded, build side on every rank."""
    parts, steps = partial_plan(aggs)
    part = (local or local_join_group)(td, build_t, probe_t, pred, lkey, rkey, keys, parts)
    return exchange_and_merge(part, keys, parts, steps, strategy, group, device)
