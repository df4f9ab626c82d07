"""td_gpu_splay_load: a splayed table read straight into HBM; a query over
it uploads nothing and matches the oracle."""
import ctypes as C

import numpy as np
import pytest

import oracle
from teide_b200.pipelines import readme_group
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
