"""Failure paths on the GPU, made on the host: the device-memory limit turns
an allocation failure into TD_ERR_OOM and the context stays usable; td_cancel
before td_execute is cleared by it (Teide resets the flag on entry), and a
cancel racing running queries yields either a correct result or
TD_ERR_CANCEL, never a wrong one."""
import ctypes as C
import threading

import numpy as np
import pytest

import oracle
from teide_b200.pipelines import readme_group
from teide_b200.td import OP_SUM, TdError

pytestmark = pytest.mark.gpu

TD_ERR_OOM, TD_ERR_CANCEL = 1, 11


def _table(gpu, n=2_000_000, seed=9):
    r = np.random.default_rng(seed)
    d = {"flag": r.integers(0, 4, n, dtype=np.int64), "region": r.integers(0, 64, n, dtype=np.int64),
         "amount": r.random(n) * 1000}
    return d, gpu.table(d)


def _want(d):
    return oracle.group({"region": d["region"]}, [(OP_SUM, "amount", d["amount"])], mask=d["flag"] == 0)


def _stats(gpu):
    class St(C.Structure):
        _fields_ = [("h2d", C.c_uint64), ("d2h", C.c_uint64), ("calls", C.c_uint64), ("live", C.c_uint64),
                    ("peak", C.c_uint64), ("gm", C.c_int32), ("jm", C.c_int32), ("fused", C.c_int32),
                    ("pad", C.c_int32)]
    s = St()
    gpu.lib.td_gpu_last_stats(C.byref(s))
    return s


def test_memory_limit_gives_oom_and_recovers(gpu):
    d, t = _table(gpu)
    L = gpu.lib
    L.td_gpu_set_mem_limit.argtypes = [C.c_size_t]
    try:
        readme_group(gpu, t, ("flag", "eq", 0), ["region"], [(OP_SUM, "amount")])   # warm caches
        live0 = _stats(gpu).live                      # device bytes held after a good query
        L.td_gpu_trim()
        L.td_gpu_set_mem_limit(64 << 10)              # far below the 48 MB upload
        with pytest.raises(TdError) as e:
            readme_group(gpu, t, ("flag", "eq", 0), ["region"], [(OP_SUM, "amount")])
        assert e.value.code == TD_ERR_OOM
        L.td_gpu_set_mem_limit(0)
        got = readme_group(gpu, t, ("flag", "eq", 0), ["region"], [(OP_SUM, "amount")])
        want = _want(d)
        assert np.array_equal(got["region"], want["region"])
        assert np.allclose(got["amount_sum"], want["amount_sum"], rtol=1e-12)
        assert _stats(gpu).live == live0              # the failed query left nothing allocated
    finally:
        L.td_gpu_set_mem_limit(0)
        gpu.release(t)


def test_cancel_before_execute_is_cleared(gpu):
    d, t = _table(gpu, n=300_000)
    try:
        gpu.lib.td_cancel()
        got = readme_group(gpu, t, ("flag", "eq", 0), ["region"], [(OP_SUM, "amount")])
        assert np.array_equal(got["region"], _want(d)["region"])
    finally:
        gpu.release(t)


def test_cancel_racing_queries_never_corrupts(gpu):
    d, t = _table(gpu)
    want = _want(d)
    stop = threading.Event()

    def canceller():
        while not stop.is_set():
            gpu.lib.td_cancel()

    th = threading.Thread(target=canceller)
    th.start()
    outcomes = []
    try:
        for _ in range(30):
            try:
                got = readme_group(gpu, t, ("flag", "eq", 0), ["region"], [(OP_SUM, "amount")])
                assert np.array_equal(got["region"], want["region"])
                assert np.allclose(got["amount_sum"], want["amount_sum"], rtol=1e-12)
                outcomes.append("ok")
            except TdError as e:
                assert e.code == TD_ERR_CANCEL
                outcomes.append("cancel")
    finally:
        stop.set()
        th.join()
    got = readme_group(gpu, t, ("flag", "eq", 0), ["region"], [(OP_SUM, "amount")])   # usable afterwards
    assert np.array_equal(got["region"], want["region"])
    gpu.release(t)
    assert len(outcomes) == 30


def _upsert(gpu):
    L = gpu.lib
    L.tdg_hash_upsert.restype = C.c_int32
    L.tdg_hash_upsert.argtypes = [C.c_void_p, C.c_void_p, C.c_uint64, C.c_int32, C.c_void_p, C.c_int64,
                                  C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]
    return L.tdg_hash_upsert


def test_hash_wait_limit_returns_error(gpu):
    """A slot left in state 1 ("being written") by a writer that never
    publishes: the readers give up after their poll limit and the call
    returns TD_ERR_IO instead of hanging.  The table is seeded on the host
    with every slot in state 1, so each key's first probe meets one; the
    same context then serves a normal upsert."""
    import torch
    TD_ERR_IO = 8
    up = _upsert(gpu)
    dev = torch.device("cuda", int(__import__("os").environ.get("TD_GPU_DEVICE", "0")))
    cap, n = 64, 100
    kv = torch.arange(n, dtype=torch.int64, device=dev) * 7919
    keys = torch.zeros(cap, dtype=torch.int64, device=dev)
    slot = torch.empty(n, dtype=torch.int64, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    state = torch.ones(cap, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    st = up(state.data_ptr(), keys.data_ptr(), cap, 1, kv.data_ptr(), n, 1000, slot.data_ptr(), err.data_ptr(),
            None)
    assert st == TD_ERR_IO
    assert (slot.cpu() == -1).all()
    # the context still works: an empty table takes every key, each once
    state.zero_()
    cap2 = 256
    state2 = torch.zeros(cap2, dtype=torch.int32, device=dev)
    keys2 = torch.zeros(cap2, dtype=torch.int64, device=dev)
    torch.cuda.synchronize()
    st = up(state2.data_ptr(), keys2.data_ptr(), cap2, 1, kv.data_ptr(), n, 0, slot.data_ptr(), err.data_ptr(),
            None)
    assert st == 0
    s = slot.cpu().numpy()
    assert (s >= 0).all() and len(np.unique(s)) == n
    assert np.array_equal(np.sort(keys2.cpu().numpy()[s]), np.sort(kv.cpu().numpy()))
    assert (state2.cpu().numpy()[s] == 2).all()
    # a full table reports TD_ERR_RANGE
    st = up(state2.data_ptr(), keys2.data_ptr(), 64, 1, (kv + 1).data_ptr(), n, 0, slot.data_ptr(),
            err.data_ptr(), None)
    assert st == 3                                  # TD_ERR_RANGE


def test_cancel_stops_the_persistent_batch_kernel(gpu, tmp_path, monkeypatch):
    """td_cancel while td_execute_batch runs: the persistent kernel polls the
    cancel word between work items and takes no further item, and the call
    returns TD_ERR_CANCEL -- or, when the cancel came too late, the whole
    correct result.  The batch works normally afterwards."""
    import os
    import sys
    sys.path.insert(0, os.path.dirname(__file__))
    from test_batch_gpu import run_batch
    from teide_b200 import workloads
    monkeypatch.setenv("TD_TUNE_CACHE", str(tmp_path / "tune.json"))
    rows, ks = workloads.batch_shapes(n_queries=256, seed=91, rows=(50_000, 400_000), groups=(16, 20_000))
    tables = [gpu.table(workloads.batch_query(int(r), int(k), seed=3000 + i)) for i, (r, k) in enumerate(zip(rows, ks))]
    try:
        want = run_batch(gpu, tables)
        stop = threading.Event()

        def canceller():
            while not stop.is_set():
                gpu.lib.td_cancel()

        th = threading.Thread(target=canceller)
        th.start()
        outcomes = []
        try:
            for _ in range(20):
                try:
                    got = run_batch(gpu, tables)
                    for k in want:
                        assert np.array_equal(got[k], want[k]) or got[k].dtype.kind == "f", k
                    outcomes.append("ok")
                except TdError as e:
                    assert e.code == TD_ERR_CANCEL
                    outcomes.append("cancel")
        finally:
            stop.set()
            th.join()
        assert "cancel" in outcomes
        again = run_batch(gpu, tables)
        for k in want:
            if want[k].dtype.kind == "f":
                assert np.allclose(again[k], want[k], rtol=1e-12, atol=0), k
            else:
                assert np.array_equal(again[k], want[k]), k
    finally:
        for t in tables:
            gpu.release(t)
