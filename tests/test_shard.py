"""Row-sharded group-by and join + group-by on CPU ranks (gloo, world size
2): the exchange of partial results.  Each rank's partial result comes from
the oracle over its own shard, and the merge of the exchanged rows is the
oracle's group-by of them (the product runs td_execute_device on each GPU and
merges with the library's own group-by, which needs a GPU and is tested in
tests/test_shard_gpu.py); the merged result must equal the oracle over all
rows."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle
from teide_b200.td import OP_AVG, OP_COUNT, OP_MAX, OP_MIN, OP_SUM

AGGS = [(OP_COUNT, "v1"), (OP_SUM, "v1"), (OP_MIN, "v1"), (OP_MAX, "v1"), (OP_AVG, "v2")]


def _data(n=200_000, nkeys=50_000, seed=3):
    r = np.random.default_rng(seed)
    return {"k1": r.integers(0, nkeys, n, dtype=np.int64), "k2": r.integers(0, 3, n, dtype=np.int64),
            "v1": r.integers(-1000, 1000, n, dtype=np.int64), "v2": r.standard_normal(n)}


def _oracle_merge(keys, vals, ops):
    """Rows of partial results merged by the oracle's group-by (SUM of the
    partial SUMs and COUNTs, MIN / MAX of the MINs / MAXs), ascending by key."""
    import torch
    kn = [f"k{j}" for j in range(keys.shape[1])]
    kd = {n: keys[:, j].numpy() for j, n in enumerate(kn)}
    if not kn:
        kd = {"k": np.zeros(keys.shape[0], np.int64)}
    aggs = [(OP_SUM if op == OP_COUNT else op, f"v{i}", v.numpy()) for i, (v, op) in enumerate(zip(vals, ops))]
    g = oracle.group(kd, aggs)
    uk = torch.as_tensor(np.stack([g[n] for n in kn], 1)) if kn else torch.zeros((len(g["k"]), 0), dtype=torch.int64)
    sfx = {OP_SUM: "_sum", OP_MIN: "_min", OP_MAX: "_max"}
    return uk, [torch.as_tensor(g[f"v{i}{sfx[a]}"]) for i, (a, _, _) in enumerate(aggs)]


def _oracle_local(keys):
    def local(td, shard, pred, _keys, parts):
        m = shard["v1"] > pred[2] if pred else None
        return oracle.group({k: shard[k] for k in keys},
                            [(op, c, None if op == OP_COUNT else shard[c]) for op, c in parts], mask=m)
    return local


def _rank(rank, world, port, keys, strategy, pred, q):
    import torch.distributed as dist
    from teide_b200 import shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        d = _data()
        n = len(d["v1"])
        lo, hi = n * rank // world, n * (rank + 1) // world
        part = {k: v[lo:hi] for k, v in d.items()}
        out = shard.sharded_group(None, part, keys, AGGS, pred=pred, strategy=strategy, device="cpu",
                                  local=_oracle_local(keys), merge=_oracle_merge)
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("strategy", ["gather", "alltoall"])
@pytest.mark.parametrize("keys", [["k1"], ["k1", "k2"]])
def test_sharded_group_matches_oracle(strategy, keys):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world, port, pred = 2, _free_port(), ("v1", "gt", -100)
    ps = [ctx.Process(target=_rank, args=(r, world, port, keys, strategy, pred, q)) for r in range(world)]
    for p in ps:
        p.start()
    outs = dict(q.get(timeout=120) for _ in range(world))
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    d = _data()
    want = oracle.group({k: d[k] for k in keys},
                        [(op, c, None if op == OP_COUNT else d[c]) for op, c in AGGS], mask=d["v1"] > -100)
    if strategy == "gather":
        got = outs[0]
        for k in got:                                   # every rank holds the whole result
            assert np.array_equal(got[k], outs[1][k]) or got[k].dtype.kind == "f"
    else:                                               # disjoint owner shares
        assert not set(map(tuple, np.stack([outs[0][k] for k in keys], 1).tolist())) & \
            set(map(tuple, np.stack([outs[1][k] for k in keys], 1).tolist()))
        got = {k: np.concatenate([outs[0][k], outs[1][k]]) for k in outs[0]}
        got = oracle.canonical(got, by=keys)
    assert list(got) == list(want)
    for k in want:
        if want[k].dtype.kind == "f":
            assert np.allclose(got[k], want[k], rtol=1e-12, atol=1e-12), k
        else:
            assert np.array_equal(got[k], want[k]), k


JAGGS = [(OP_SUM, "price"), (OP_COUNT, "price"), (OP_AVG, "price"), (OP_MAX, "qty")]


def _join_local(td, build, probe, pred, lkey, rkey, keys, parts):
    m = probe[pred[0]] > pred[2]
    li, ri = oracle.join_pairs([probe[lkey]], [build[rkey]], 0, m)
    j = {**{k: v[li] for k, v in probe.items()}, **{k: v[ri] for k, v in build.items() if k != rkey}}
    return oracle.group({k: j[k] for k in keys}, [(op, c, None if op == OP_COUNT else j[c]) for op, c in parts])


def _join_rank(rank, world, port, strategy, q):
    import torch.distributed as dist
    from teide_b200 import shard, workloads
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        b, p = workloads.join_tables(n_build=20_000, n_probe=300_000, seed=17)
        n = len(p["fk"])
        lo, hi = n * rank // world, n * (rank + 1) // world
        shard_p = {k: v[lo:hi] for k, v in p.items()}
        out = shard.sharded_join_group(None, b, shard_p, ("qty", "gt", 10), "fk", "pk", ["cat"], JAGGS,
                                       strategy=strategy, device="cpu", local=_join_local, merge=_oracle_merge)
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("strategy", ["gather", "alltoall"])
def test_sharded_join_group_matches_oracle(strategy):
    """Probe rows sharded over two ranks, the build side on both: the merged
    filter -> join -> group-by equals the oracle's over all probe rows."""
    from teide_b200 import workloads
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    world, port = 2, _free_port()
    ps = [ctx.Process(target=_join_rank, args=(r, world, port, strategy, q)) for r in range(world)]
    for p in ps:
        p.start()
    outs = dict(q.get(timeout=120) for _ in range(world))
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    b, p = workloads.join_tables(n_build=20_000, n_probe=300_000, seed=17)
    j = oracle.join(p, b, ["fk"], ["pk"], 0, p["qty"] > 10)
    want = oracle.group({"cat": j["cat"]}, [(op, c, None if op == OP_COUNT else j[c]) for op, c in JAGGS])
    got = outs[0] if strategy == "gather" else oracle.canonical(
        {k: np.concatenate([outs[0][k], outs[1][k]]) for k in outs[0]}, by=["cat"])
    assert list(got) == list(want)
    for k in want:
        if want[k].dtype.kind == "f":
            assert np.allclose(got[k], want[k], rtol=1e-12, atol=0), k
        else:
            assert np.array_equal(got[k], want[k]), k


def test_partial_plan_avg_becomes_sum_and_count():
    from teide_b200.shard import partial_plan
    parts, steps = partial_plan([(OP_AVG, "x"), (OP_SUM, "x"), (OP_COUNT, "y")])
    assert parts == [(OP_SUM, "x"), (OP_COUNT, "x"), (OP_COUNT, "y")]
    assert steps == [("avg", 0, 1), ("id", 0), ("id", 2)]
