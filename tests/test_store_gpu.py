"""td_gpu_splay_load: a splayed table read straight into HBM; a query over
it uploads nothing and matches the oracle."""
import ctypes as C

import numpy as np
import pytest

import oracle
from teide_b200.pipelines import f64_tolerance_ok, readme_group
from teide_b200 import workloads
from teide_b200.td import OP_SUM

pytestmark = pytest.mark.gpu


class St(C.Structure):
    _fields_ = [("h2d", C.c_uint64), ("d2h", C.c_uint64), ("calls", C.c_uint64), ("live", C.c_uint64),
                ("peak", C.c_uint64), ("gm", C.c_int32), ("jm", C.c_int32), ("fused", C.c_int32),
                ("pad", C.c_int32)]


def test_splayed_table_loads_resident(gpu, tmp_path):
    L = gpu.lib
    L.td_gpu_splay_load.restype = C.c_void_p
    L.td_gpu_splay_load.argtypes = [C.c_char_p]
    L.td_gpu_unpin.argtypes = [C.c_void_p]
    d = workloads.readme_table(n=2_000_000, seed=61)
    t = gpu.table(d)
    dirp = str(tmp_path / "readme")
    assert L.td_splay_save(t, dirp.encode(), None) == 0
    gpu.release(t)
    r = gpu.check(L.td_gpu_splay_load(dirp.encode()), "td_gpu_splay_load")
    try:
        got = readme_group(gpu, r, ("flag", "eq", 0), ["region"], [(OP_SUM, "amount")])
        s = St()
        L.td_gpu_last_stats(C.byref(s))
        assert s.h2d == 0                                      # every column was already on the device
        m = d["flag"] == 0
        want = oracle.group({"region": d["region"][m]}, [(OP_SUM, "amount", d["amount"][m])])
        assert np.array_equal(got["region"], want["region"])
        assert np.allclose(got["amount_sum"], want["amount_sum"], rtol=1e-12)
    finally:
        L.td_gpu_unpin(r)
        gpu.release(r)


def test_partitioned_db_loads_resident(gpu, tmp_path):
    L = gpu.lib
    L.td_gpu_part_load.restype = C.c_void_p
    L.td_gpu_part_load.argtypes = [C.c_char_p, C.c_char_p]
    L.td_gpu_unpin.argtypes = [C.c_void_p]
    parts = {}
    for i, day in enumerate(["2024.03.01", "2024.03.02", "2024.03.03"]):
        d = workloads.readme_table(n=300_000 + 1000 * i, seed=70 + i)
        t = gpu.table(d)
        (tmp_path / day).mkdir()
        assert L.td_splay_save(t, str(tmp_path / day / "t").encode(), None) == 0
        gpu.release(t)
        parts[day] = d
    r = gpu.check(L.td_gpu_part_load(str(tmp_path).encode(), b"t"), "td_gpu_part_load")
    try:
        got = readme_group(gpu, r, ("flag", "eq", 0), ["region"], [(OP_SUM, "amount")])
        s = St()
        L.td_gpu_last_stats(C.byref(s))
        assert s.h2d == 0
        d = {k: np.concatenate([parts[p][k] for p in sorted(parts)]) for k in ("flag", "region", "amount")}
        m = d["flag"] == 0
        want = oracle.group({"region": d["region"][m]}, [(OP_SUM, "amount", d["amount"][m])])
        assert np.array_equal(got["region"], want["region"])
        assert np.allclose(got["amount_sum"], want["amount_sum"], rtol=1e-12)
    finally:
        L.td_gpu_unpin(r)
        gpu.release(r)


# ---- partitioned tables -----------------------------------------------------------------

BIG_PARTS = {"2024.01.02": 400_000, "2023.12.31": 700_000, "2024.01.01": 0, "2024.01.10": 90_000,
             "2024.02.29": 250_000}


@pytest.mark.parametrize("pinned", [False, True], ids=["uploaded", "resident"])
def test_parted_group_by(gpu, tmp_path, pinned):
    """Group-bys over td_read_parted's partitioned table: by the MAPCOMMON
    partition key (expanded over the rows on the device), by a parted column
    (its segments laid end to end on the device), and by both -- each equal
    to the oracle over the partitions' rows.  Resident (td_gpu_pin), a second
    query uploads nothing."""
    import sys
    import os
    sys.path.insert(0, os.path.dirname(__file__))
    from test_store import PARTED_QUERIES, _parted_db, parted_group, parted_want
    cols = _parted_db(gpu, tmp_path, BIG_PARTS)
    order = sorted(BIG_PARTS)
    L = gpu.lib
    if pinned:
        L.td_read_parted.restype = C.c_void_p
        L.td_read_parted.argtypes = [C.c_char_p, C.c_char_p]
        L.td_gpu_pin.argtypes = [C.c_void_p]
        L.td_gpu_unpin.argtypes = [C.c_void_p]
        t = gpu.check(L.td_read_parted(str(tmp_path).encode(), b"trades"), "read_parted")
        assert L.td_gpu_pin(t) == 0
    for keys, aggs in PARTED_QUERIES:
        if pinned:
            g = gpu.graph(t)
            try:
                r = g.execute(g.group([g.scan(k) for k in keys], [op for op, _ in aggs],
                                      [g.scan(c) for _, c in aggs]), optimize=False)
            finally:
                g.free()
            s = St()
            L.td_gpu_last_stats(C.byref(s))
            assert s.h2d == 0, keys                   # every column resident, flattened once
            got = gpu.table_dict(r)
            gpu.release(r)
        else:
            got = parted_group(gpu, tmp_path, keys, aggs)
        got = oracle.canonical(got, by=keys)
        want = parted_want(cols, order, keys, aggs)
        assert list(got) == list(want), keys
        absd = {p: {**cols[p], "px": np.abs(cols[p]["px"])} for p in order}
        bounds = parted_want(absd, order, keys, aggs)            # sum |px| (or its mean) per group
        for k in want:
            if want[k].dtype.kind == "f":
                assert f64_tolerance_ok(got[k], want[k], bounds[k]), (keys, k)
            else:
                assert got[k].dtype == want[k].dtype and np.array_equal(got[k], want[k]), (keys, k)
    if pinned:
        L.td_gpu_unpin(t)
        gpu.release(t)


def test_mapped_splayed_table_queries(gpu, tmp_path):
    """A splayed table opened with td_read_splayed (every column mapped from
    its file, copy-on-write) uploads from the mapped pages and groups like
    the oracle; pinned, the next query uploads nothing."""
    L = gpu.lib
    L.td_gpu_pin.argtypes = [C.c_void_p]
    L.td_gpu_unpin.argtypes = [C.c_void_p]
    d = workloads.readme_table(n=3_000_001, seed=63)
    t = gpu.table(d)
    dirp = str(tmp_path / "mapped")
    assert L.td_splay_save(t, dirp.encode(), None) == 0
    gpu.release(t)
    r = gpu.check(L.td_read_splayed(dirp.encode(), None), "td_read_splayed")
    try:
        m = d["flag"] == 0
        want = oracle.group({"region": d["region"][m]}, [(OP_SUM, "amount", d["amount"][m])])
        absum = oracle.group({"region": d["region"][m]}, [(OP_SUM, "amount", np.abs(d["amount"][m]))])
        got = readme_group(gpu, r, ("flag", "eq", 0), ["region"], [(OP_SUM, "amount")])
        assert np.array_equal(got["region"], want["region"])
        assert f64_tolerance_ok(got["amount_sum"], want["amount_sum"], absum["amount_sum"])
        assert L.td_gpu_pin(r) == 0
        got = readme_group(gpu, r, ("flag", "eq", 0), ["region"], [(OP_SUM, "amount")])
        s = St()
        L.td_gpu_last_stats(C.byref(s))
        assert s.h2d == 0
        assert np.array_equal(got["region"], want["region"])
    finally:
        L.td_gpu_unpin(r)
        gpu.release(r)
