"""td_sort_op / td_head on the GPU (tdg_sort_perm + tdg_gather) against the
oracle: the shared cases Teide pins, plus sizes past one radix tile, empty
and one-row tables, a limit beyond the row count, and HEAD without a sort."""
import numpy as np
import pytest

import oracle
import sort_cases
from teide_b200.td import BOOL, I16, U8

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", sort_cases.ALL, ids=lambda c: c.__name__)
def test_sort_matches_oracle(gpu, case):
    got, want = case(gpu)
    sort_cases.same(got, want)


@pytest.mark.parametrize("case", ["a", "b", "c", "d"])
def test_sort_golden(gpu, case):
    """Teide's own row order (tests/golden/sort_small.npz, made by running
    Teide) reproduced through td_sort_op on the device, bit for bit."""
    import os
    with np.load(os.path.join(os.path.dirname(__file__), "golden", "sort_small.npz")) as z:
        zz = {k: z[k] for k in z.files}
    cols = {k[len(case) + 4:]: v for k, v in zz.items() if k.startswith(case + "_in_")}
    want = {k[len(case) + 5:]: v for k, v in zz.items() if k.startswith(case + "_out_")}
    keys = []
    for spec in zz[case + "_keys"]:
        name, desc, nf = str(spec).split(":")
        keys.append((name, bool(int(desc)), None if int(nf) < 0 else bool(int(nf))))
    tags = {"b": BOOL, "h": I16, "u": U8} if case == "d" else {}
    t = gpu.table({k: ((v, tags[k]) if k in tags else v) for k, v in cols.items()})
    try:
        got = sort_cases._run(gpu, t, keys)
    finally:
        gpu.release(t)
    sort_cases.same(sort_cases._bits(got), sort_cases._bits(want))


def test_small_int_and_zero_keys_many_tiles(gpu):
    """I16 DESC, U8, then F64 with both zeros (equal under several keys) over
    300K rows: many radix tiles, 16- and 8-bit digit counts."""
    n = 300_001
    r = np.random.default_rng(31)
    d = {"h": r.integers(-2**15, 2**15, n).astype(np.int16), "u": r.integers(0, 256, n).astype(np.uint8),
         "f": np.where(r.integers(0, 2, n) == 1, -0.0, 0.0), "i": np.arange(n)}
    t = gpu.table({"h": (d["h"], I16), "u": (d["u"], U8), "f": d["f"], "i": d["i"]})
    try:
        keys = [("h", True, None), ("u", False, None), ("f", False, None)]
        sort_cases.same(sort_cases._bits(sort_cases._run(gpu, t, keys)), sort_cases._bits(oracle.sort(d, keys)))
    finally:
        gpu.release(t)


@pytest.mark.parametrize("n", [0, 1, 63, 4097, 1_000_003])
def test_sort_sizes(gpu, n):
    r = np.random.default_rng(n)
    d = {"k": r.integers(-2**62, 2**62, n), "j": r.integers(0, 3, n), "i": np.arange(n)}
    t = gpu.table(d)
    try:
        keys = [("j", True, None), ("k", False, None)]
        sort_cases.same(sort_cases._run(gpu, t, keys), oracle.sort(d, keys))
    finally:
        gpu.release(t)


def test_limit_beyond_rows_and_plain_head(gpu):
    d = {"k": np.array([5, 3, 9, 1], dtype=np.int64), "i": np.arange(4)}
    t = gpu.table(d)
    try:
        sort_cases.same(sort_cases._run(gpu, t, [("k", False, None)], limit=10),
                        oracle.sort(d, [("k", False, None)]))
        g = gpu.graph(t)
        try:
            r = g.execute(g.head(g.const_table(t), 2), optimize=False)
        finally:
            g.free()
        out = gpu.table_dict(r)
        gpu.release(r)
        assert np.array_equal(out["k"], d["k"][:2]) and np.array_equal(out["i"], d["i"][:2])
    finally:
        gpu.release(t)


def test_sort_of_group_without_result_mirrors(gpu, monkeypatch):
    """With result mirrors off the group result the sort reads is copied to
    the host and uploaded again: same answer."""
    monkeypatch.setenv("TD_GPU_NO_RESULT_MIRROR", "1")
    got, want = sort_cases.sort_of_group(gpu)
    sort_cases.same(got, want)
