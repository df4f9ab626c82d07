"""Column files and splayed tables in Teide's on-disk format: a column saved
by either library is byte-identical to the other's and loads in both; slices
save as their own rows; splayed tables and the symbol file round-trip."""
import os

import numpy as np
import pytest

from teide_b200.td import I16, I32, U8, BOOL

COLS = {
    "i64": (np.arange(-500, 500, dtype=np.int64) * 7919, None),
    "f64": (np.linspace(-3, 3, 999), None),
    "i32": (np.arange(1000, dtype=np.int32) - 300, I32),
    "i16": (np.arange(777, dtype=np.int16), I16),
    "u8": ((np.arange(300) % 256).astype(np.uint8), U8),
    "b": (np.arange(50) % 3 == 0, BOOL),
    "empty": (np.zeros(0, dtype=np.int64), None),
}


def _vec(td, arr, typ):
    return td.vec(arr, typ) if typ is not None else td.vec(arr)


@pytest.mark.parametrize("name", list(COLS))
def test_column_files_match_reference_and_cross_load(td, ref, tmp_path, name):
    arr, typ = COLS[name]
    ours, theirs = str(tmp_path / "ours.col"), str(tmp_path / "theirs.col")
    a, b = _vec(td, arr, typ), _vec(ref, arr, typ)
    try:
        assert td.lib.td_col_save(a, ours.encode()) == 0
        assert ref.lib.td_col_save(b, theirs.encode()) == 0
        assert open(ours, "rb").read() == open(theirs, "rb").read()
        for lib, path in ((td, theirs), (ref, ours)):
            v = lib.check(lib.lib.td_col_load(path.encode()), "td_col_load")
            got = lib.to_numpy(v)
            assert np.array_equal(got.astype(arr.dtype) if arr.dtype == np.bool_ else got, arr)
            lib.release(v)
    finally:
        td.release(a)
        ref.release(b)


def test_sym_column_widths(td, tmp_path):
    for w in range(4):
        ids = np.arange(0, 60) % (1 << (8 << w) if w < 3 else 1 << 40)
        v = td.sym_vec(ids, w)
        p = str(tmp_path / f"s{w}.col").encode()
        assert td.lib.td_col_save(v, p) == 0
        r = td.check(td.lib.td_col_load(p), "load")
        assert np.array_equal(td.to_numpy(r), td.to_numpy(v))
        td.release(r)
        td.release(v)


def test_slice_saves_its_rows(td, tmp_path):
    td.lib.td_vec_slice.restype = td.lib.td_col_load.restype
    td.lib.td_vec_slice.argtypes = [td.lib.td_col_load.restype, __import__("ctypes").c_int64,
                                    __import__("ctypes").c_int64]
    arr = np.arange(100, dtype=np.int64) * 3
    v = td.vec(arr)
    s = td.check(td.lib.td_vec_slice(v, 10, 25), "slice")
    p = str(tmp_path / "slice.col").encode()
    assert td.lib.td_col_save(s, p) == 0
    r = td.check(td.lib.td_col_load(p), "load")
    assert np.array_equal(td.to_numpy(r), arr[10:35])
    for x in (r, s, v):
        td.release(x)


def test_splayed_table_and_symbols_round_trip(td, tmp_path):
    d = {"k": np.arange(1000, dtype=np.int64) % 17, "v": np.linspace(0, 1, 1000)}
    t = td.table(d)
    dirp, symp = str(tmp_path / "tbl"), str(tmp_path / "sym")
    try:
        assert td.lib.td_splay_save(t, dirp.encode(), symp.encode()) == 0
        assert sorted(os.listdir(dirp)) == [".d", "k", "v"]
        assert open(symp, "rb").read(4) == b"TSYM"
        n_before = td.lib.td_sym_count()
        assert td.lib.td_sym_load(symp.encode()) == 0          # every name is already interned
        assert td.lib.td_sym_count() == n_before
        r = td.check(td.lib.td_splay_load(dirp.encode()), "splay load")
        got = td.table_dict(r)
        td.release(r)
        assert list(got) == ["k", "v"]
        assert np.array_equal(got["k"], d["k"]) and np.array_equal(got["v"], d["v"])
    finally:
        td.release(t)


def test_corrupt_files_are_refused(td, tmp_path):
    p = tmp_path / "bad.col"
    p.write_bytes(b"\0" * 10)
    r = td.lib.td_col_load(str(p).encode())
    assert r is not None and r < 32                            # TD_ERR_PTR(corrupt): too short for a header
    v = td.vec(np.arange(10, dtype=np.int64))
    good = tmp_path / "good.col"
    assert td.lib.td_col_save(v, str(good).encode()) == 0
    good_bytes = good.read_bytes()
    p.write_bytes(good_bytes[:-8])                              # one element short
    r = td.lib.td_col_load(str(p).encode())
    assert r is not None and r < 32                            # TD_ERR_PTR(corrupt)
    td.release(v)


PARTS = {"2024.01.02": 700, "2023.12.31": 1300, "2024.01.01": 0, "2024.01.10": 55}


def _write_db(lib, root, parts, seed=9):
    r = np.random.default_rng(seed)
    cols = {}
    for name, n in parts.items():
        d = {"k": r.integers(0, 40, n), "px": r.standard_normal(n), "q": r.integers(-9, 9, n).astype(np.int32)}
        cols[name] = d
        t = lib.table({"k": d["k"], "px": d["px"], "q": (d["q"], I32)})
        os.makedirs(f"{root}/{name}", exist_ok=True)             # td_splay_save makes only the leaf
        assert lib.lib.td_splay_save(t, f"{root}/{name}/trades".encode(), None) == 0
        lib.release(t)
    os.makedirs(f"{root}/notes", exist_ok=True)                  # not a partition name: skipped
    return cols


def test_partitioned_db_matches_reference(td, ref, tmp_path):
    for p in ("ours", "theirs"):
        os.makedirs(tmp_path / p)
    want = _write_db(td, tmp_path / "ours", PARTS)
    _write_db(ref, tmp_path / "theirs", PARTS)
    r1 = td.check(td.lib.td_part_load(str(tmp_path / "ours").encode(), b"trades"), "part load")
    r2 = ref.check(ref.lib.td_part_load(str(tmp_path / "theirs").encode(), b"trades"), "part load")
    ours, theirs = td.table_dict(r1), ref.table_dict(r2)
    td.release(r1)
    ref.release(r2)
    assert list(ours) == list(theirs) == ["k", "px", "q"]
    order = sorted(PARTS)
    for c in ours:
        cat = np.concatenate([want[p][c] for p in order])
        assert np.array_equal(ours[c], theirs[c]), c
        assert np.array_equal(ours[c], cat), c


# ---- partitioned tables (td_read_parted) -------------------------------------------

def _parted_db(lib, root, parts, seed=9):
    cols = _write_db(lib, root, parts, seed)
    assert lib.lib.td_sym_save(f"{root}/sym".encode()) == 0
    return cols


def _col_info(lib, p):
    """(type, attrs, len, element pointers) of a vector whose elements are td_t pointers."""
    import ctypes as C
    typ, attrs, n = lib.header(p)
    ptrs = [C.c_void_p.from_address(p + 32 + 8 * i).value for i in range(n)]
    return typ, attrs, n, ptrs


def test_read_parted_matches_reference(td, ref, tmp_path):
    """The partitioned table of both libraries over the same database: the
    MAPCOMMON column first (DATE keys of the YYYY.MM.DD directories, their row
    counts), then one parted column per column, segments in name order."""
    import ctypes as C
    out = {}
    for name, lib in (("ours", td), ("theirs", ref)):
        os.makedirs(tmp_path / name)
        want = _parted_db(lib, tmp_path / name, PARTS)
        lib.lib.td_read_parted.restype = C.c_void_p
        lib.lib.td_read_parted.argtypes = [C.c_char_p, C.c_char_p]
        lib.lib.td_parted_nrows.restype = C.c_int64
        lib.lib.td_parted_nrows.argtypes = [C.c_void_p]
        t = lib.check(lib.lib.td_read_parted(str(tmp_path / name).encode(), b"trades"), "read_parted")
        L = lib.lib
        cols = []
        for j in range(L.td_table_ncols(t)):
            c = L.td_table_get_col_idx(t, j)
            typ, attrs, n, ptrs = _col_info(lib, c)
            entry = {"name": lib.sym_name(L.td_table_col_name(t, j)), "type": typ, "n": n,
                     "rows": L.td_parted_nrows(c)}
            if typ == 64:                                  # MAPCOMMON: key values, row counts
                entry["attrs"] = attrs
                entry["keys"] = lib.vec_view(ptrs[0]).copy().tolist()
                entry["counts"] = lib.vec_view(ptrs[1]).copy().tolist()
            else:
                entry["segs"] = [lib.vec_view(q).copy() for q in ptrs]
            cols.append(entry)
        out[name] = (cols, L.td_table_nrows(t), want)
        lib.release(t)
    (a, na, want), (b, nb, _) = out["ours"], out["theirs"]
    order = sorted(PARTS)
    assert na == nb == sum(PARTS.values())
    assert [c["name"] for c in a] == [c["name"] for c in b] == ["date", "k", "px", "q"]
    for x, y in zip(a, b):
        assert x["type"] == y["type"] and x["n"] == y["n"] and x["rows"] == y["rows"], x["name"]
        if x["type"] == 64:
            assert x["attrs"] == y["attrs"] == 1 and x["keys"] == y["keys"] and x["counts"] == y["counts"]
            assert x["counts"] == [PARTS[p] for p in order]
        else:
            for p, s1, s2 in zip(order, x["segs"], y["segs"]):
                assert np.array_equal(s1, s2) and np.array_equal(s1, want[p][x["name"]]), (x["name"], p)


PARTED_QUERIES = [
    (["date"], [(50, "px"), (54, "px"), (53, "k")]),            # the partition key alone
    (["k"], [(50, "q"), (52, "px"), (55, "px")]),               # a parted column
    (["date", "k"], [(50, "px"), (54, "q")]),                   # both
]


def parted_want(cols, order, keys, aggs):
    """The oracle's group-by over the partitions' rows, the partition key
    (days since 2000-01-01 of each YYYY.MM.DD name) repeated over its rows."""
    import datetime
    import oracle
    flat = {c: np.concatenate([cols[p][c] for p in order]) for c in ("k", "px", "q")}
    days = [(datetime.date(int(p[:4]), int(p[5:7]), int(p[8:])) - datetime.date(2000, 1, 1)).days for p in order]
    flat["date"] = np.repeat(np.array(days, np.int32), [len(cols[p]["k"]) for p in order])
    return oracle.group({k: flat[k] for k in keys}, [(op, c, None if op == 54 else flat[c]) for op, c in aggs])


def parted_group(lib, root, keys, aggs):
    import ctypes as C
    lib.lib.td_read_parted.restype = C.c_void_p
    lib.lib.td_read_parted.argtypes = [C.c_char_p, C.c_char_p]
    t = lib.check(lib.lib.td_read_parted(str(root).encode(), b"trades"), "read_parted")
    g = lib.graph(t)
    try:
        r = g.execute(g.group([g.scan(k) for k in keys], [op for op, _ in aggs], [g.scan(c) for _, c in aggs]),
                      optimize=False)
    finally:
        g.free()
    out = lib.table_dict(r)
    lib.release(r)
    lib.release(t)
    return out


@pytest.mark.parametrize("q", range(len(PARTED_QUERIES)))
def test_reference_parted_group_matches_oracle(ref, tmp_path, q):
    """Teide's own group-by over a partitioned table (its per-partition or
    concatenating path) pins the oracle's reading: the MAPCOMMON key repeated
    over each partition's rows."""
    import oracle
    keys, aggs = PARTED_QUERIES[q]
    cols = _parted_db(ref, tmp_path, PARTS)
    got = oracle.canonical(parted_group(ref, tmp_path, keys, aggs), by=keys)
    want = parted_want(cols, sorted(PARTS), keys, aggs)
    assert list(got) == list(want)
    for k in want:
        if want[k].dtype.kind == "f":
            assert np.allclose(got[k], want[k], rtol=1e-12, atol=1e-12), k
        else:
            assert np.array_equal(got[k].astype(want[k].dtype), want[k]), k


@pytest.mark.parametrize("name", ["i64", "f64", "i32", "u8", "empty"])
def test_col_mmap_matches_file_and_reference(td, ref, tmp_path, name):
    """td_col_mmap maps a column file copy-on-write: the same elements as
    td_col_load and as Teide's own td_col_mmap of the same file, mmod = 1,
    and writing an element changes the mapped vector but not the file."""
    arr, typ = COLS[name]
    path = str(tmp_path / "c.col")
    a = _vec(td, arr, typ)
    try:
        assert td.lib.td_col_save(a, path.encode()) == 0
        before = open(path, "rb").read()
        v = td.check(td.lib.td_col_mmap(path.encode()), "td_col_mmap")
        w = ref.check(ref.lib.td_col_mmap(path.encode()), "td_col_mmap (Teide)")
        got, theirs = td.to_numpy(v), ref.to_numpy(w)
        assert np.array_equal(got, theirs) and np.array_equal(got.astype(arr.dtype), arr)
        if len(arr):
            view = td.vec_view(v)                   # the mapped pages themselves
            view[0] = view[0] + 1
            assert td.to_numpy(v)[0] == got[0] + 1
        td.release(v)
        ref.release(w)
        assert open(path, "rb").read() == before
    finally:
        td.release(a)


def test_read_splayed_maps_every_column(td, tmp_path):
    """td_read_splayed gives the table td_splay_load gives, with every column
    mapped from its file; the symbol file is loaded first when named."""
    d = {"k": np.arange(5000, dtype=np.int64) % 37, "v": np.linspace(-1, 1, 5000), "n": np.arange(5000, dtype=np.int32)}
    t = td.table({"k": d["k"], "v": d["v"], "n": td.vec(d["n"], I32)})
    dirp, symp = str(tmp_path / "tbl"), str(tmp_path / "sym")
    try:
        assert td.lib.td_splay_save(t, dirp.encode(), symp.encode()) == 0
        r = td.check(td.lib.td_read_splayed(dirp.encode(), symp.encode()), "td_read_splayed")
        s = td.check(td.lib.td_splay_load(dirp.encode()), "td_splay_load")
        got, want = td.table_dict(r), td.table_dict(s)
        td.release(r)
        td.release(s)
        assert list(got) == list(want) == ["k", "v", "n"]
        for k in got:
            assert np.array_equal(got[k], want[k]), k
        assert np.array_equal(got["k"], d["k"]) and np.array_equal(got["n"], d["n"])
    finally:
        td.release(t)


def test_heap_reuses_blocks_across_threads(td):
    """Freed small blocks are kept per size and handed out again (also to
    other threads): vectors allocated, filled and released by four threads
    at once keep their own contents."""
    import threading
    from teide_b200.td import I64
    errors = []

    def work(seed):
        r = np.random.default_rng(seed)
        for _ in range(300):
            live = []
            for _ in range(8):
                n = int(r.integers(1, 20_000))
                p, view = td.vec_alloc(I64, n)
                view[:] = np.arange(n, dtype=np.int64) * seed
                live.append((p, n))
            for p, n in live:
                if not np.array_equal(td.to_numpy(p), np.arange(n, dtype=np.int64) * seed):
                    errors.append(seed)
                td.release(p)

    th = [threading.Thread(target=work, args=(s,)) for s in (3, 5, 7, 11)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errors
