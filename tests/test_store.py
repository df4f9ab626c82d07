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
