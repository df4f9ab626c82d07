"""ctypes binding of the Teide C API (include/teide/td.h).

`Td(path)` binds any shared library that exports the td.h ABI.  The product
library is libteide_b200.so (this package); the same class drives any other
build of the API, which is how the parity tests run identical DAGs on two
engines.  Helpers convert numpy arrays to td_t columns/tables and back.

Layout facts used here (all from td.h): a td_t is a 32-byte header -- type
int8 at byte 18, attrs uint8 at 19, rc uint32 at 20, len int64 at 24 -- with
elements inline from byte 32; a table's data is [schema, col_0, col_1, ...]
where schema is an I64 vector of column-name symbol ids; pointer values
below 32 encode a td_err_t.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

# type tags (td.h)
LIST, BOOL, U8, CHAR, I16, I32, I64, F64 = 0, 1, 2, 3, 4, 5, 6, 7
DATE, TIME, TIMESTAMP, GUID, TABLE, SEL, SYM = 9, 10, 11, 12, 13, 16, 20

# opcodes used by the relational path (td.h)
OP_SUM, OP_MIN, OP_MAX, OP_COUNT, OP_AVG = 50, 52, 53, 54, 55

ERRORS = ["ok", "oom", "type", "range", "length", "rank", "domain", "nyi",
          "io", "schema", "corrupt", "cancel"]

NP_OF = {BOOL: np.uint8, U8: np.uint8, CHAR: np.uint8, I16: np.int16, I32: np.int32,
         I64: np.int64, F64: np.float64, DATE: np.int32, TIME: np.int32,
         TIMESTAMP: np.int64}
SYM_NP = {0: np.uint8, 1: np.uint16, 2: np.uint32, 3: np.int64}
TYPE_OF_NP = {np.dtype(np.int64): I64, np.dtype(np.float64): F64, np.dtype(np.int32): I32,
              np.dtype(np.int16): I16, np.dtype(np.uint8): U8, np.dtype(np.bool_): BOOL}


class TdError(RuntimeError):
    def __init__(self, code: int, what: str = ""):
        self.code = code
        name = ERRORS[code] if 0 <= code < len(ERRORS) else str(code)
        super().__init__(f"td error {code} ({name}){': ' + what if what else ''}")


P = C.c_void_p


class Td:
    """Binding of one library exporting the td.h API."""

    def __init__(self, path: str):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.path = path
        self.lib = C.CDLL(path, mode=os.RTLD_LOCAL | os.RTLD_NOW)
        L = self.lib
        sig = {
            "td_heap_init": (None, []), "td_sym_init": (None, []),
            "td_heap_destroy": (None, []), "td_sym_destroy": (None, []),
            "td_vec_new": (P, [C.c_int8, C.c_int64]),
            "td_vec_from_raw": (P, [C.c_int8, P, C.c_int64]),
            "td_sym_vec_new": (P, [C.c_uint8, C.c_int64]),
            "td_table_new": (P, [C.c_int64]),
            "td_table_add_col": (P, [P, C.c_int64, P]),
            "td_table_get_col": (P, [P, C.c_int64]),
            "td_table_get_col_idx": (P, [P, C.c_int64]),
            "td_table_col_name": (C.c_int64, [P, C.c_int64]),
            "td_table_ncols": (C.c_int64, [P]), "td_table_nrows": (C.c_int64, [P]),
            "td_sym_intern": (C.c_int64, [C.c_char_p, C.c_size_t]),
            "td_sym_str": (P, [C.c_int64]),
            "td_str_ptr": (C.c_char_p, [P]), "td_str_len": (C.c_size_t, [P]),
            "td_retain": (None, [P]), "td_release": (None, [P]),
            "td_graph_new": (P, [P]), "td_graph_free": (None, [P]),
            "td_graph_add_table": (C.c_uint16, [P, P]),
            "td_scan": (P, [P, C.c_char_p]),
            "td_scan_table": (P, [P, C.c_uint16, C.c_char_p]),
            "td_const_i64": (P, [P, C.c_int64]), "td_const_f64": (P, [P, C.c_double]),
            "td_const_bool": (P, [P, C.c_bool]), "td_const_str": (P, [P, C.c_char_p]),
            "td_const_table": (P, [P, P]), "td_const_vec": (P, [P, P]),
            "td_filter": (P, [P, P, P]),
            "td_group": (P, [P, P, C.c_uint8, P, P, C.c_uint8]),
            "td_join": (P, [P, P, P, P, P, C.c_uint8, C.c_uint8]),
            "td_optimize": (P, [P, P]), "td_execute": (P, [P, P]),
            "td_sel_new": (P, [C.c_int64]), "td_sel_from_pred": (P, [P]),
            "td_sel_and": (P, [P, P]), "td_sel_recompute": (None, [P]),
            "td_cancel": (None, []),
            "td_sort_op": (P, [P, P, P, P, P, C.c_uint8]),
            "td_head": (P, [P, P, C.c_int64]),
            "td_col_save": (C.c_int, [P, C.c_char_p]), "td_col_load": (P, [C.c_char_p]),
            "td_splay_save": (C.c_int, [P, C.c_char_p, C.c_char_p]), "td_splay_load": (P, [C.c_char_p]),
            "td_sym_save": (C.c_int, [C.c_char_p]), "td_sym_load": (C.c_int, [C.c_char_p]),
            "td_part_load": (P, [C.c_char_p, C.c_char_p]),
            "td_col_mmap": (P, [C.c_char_p]), "td_read_splayed": (P, [C.c_char_p, C.c_char_p]),
        }
        for name in ("td_eq", "td_ne", "td_lt", "td_le", "td_gt", "td_ge", "td_and", "td_or",
                     "td_add", "td_sub", "td_mul", "td_div", "td_mod", "td_min2", "td_max2"):
            sig[name] = (P, [P, P, P])
        for name in ("td_not", "td_neg", "td_abs", "td_sum", "td_count", "td_avg",
                     "td_min_op", "td_max_op"):
            sig[name] = (P, [P, P])
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        L.td_heap_init()
        L.td_sym_init()

    # ---- symbols ---------------------------------------------------------------
    def sym(self, name: str) -> int:
        b = name.encode()
        return self.lib.td_sym_intern(b, len(b))

    def sym_name(self, sid: int) -> str:
        a = self.lib.td_sym_str(sid)
        if not a:
            return f"#{sid}"
        n = self.lib.td_str_len(a)
        p = self.lib.td_str_ptr(a)
        return C.string_at(p, n).decode() if n else ""

    # ---- td_t access -------------------------------------------------------------
    @staticmethod
    def check(p, what=""):
        v = p or 0
        if v < 32:
            raise TdError(v, what)
        return v

    @staticmethod
    def header(p):
        raw = C.string_at(p + 16, 16)
        typ = np.frombuffer(raw[2:3], np.int8)[0]
        attrs = raw[3]
        ln = np.frombuffer(raw[8:16], np.int64)[0]
        return int(typ), int(attrs), int(ln)

    def vec_view(self, p) -> np.ndarray:
        """numpy view of a vector's elements (valid while the vector lives)."""
        typ, attrs, n = self.header(p)
        dt = SYM_NP[attrs & 3] if typ == SYM else NP_OF[typ]
        if n == 0:
            return np.zeros(0, dt)
        buf = (C.c_char * (n * np.dtype(dt).itemsize)).from_address(p + 32)
        return np.frombuffer(buf, dt, n)

    def to_numpy(self, p) -> np.ndarray:
        return self.vec_view(p).copy()

    def atom_value(self, p):
        typ, _, _ = self.header(p)
        raw = C.string_at(p + 24, 8)
        if typ == -F64:
            return float(np.frombuffer(raw, np.float64)[0])
        if typ == -BOOL:
            return bool(raw[0])
        return int(np.frombuffer(raw, np.int64)[0])

    # ---- construction --------------------------------------------------------------
    def vec(self, arr, typ=None):
        arr = np.ascontiguousarray(arr)
        if typ is None:
            typ = TYPE_OF_NP[arr.dtype]
        if arr.dtype == np.bool_:
            arr = arr.astype(np.uint8)
        return self.check(self.lib.td_vec_from_raw(typ, arr.ctypes.data, arr.size), "vec")

    def sym_vec(self, ids, width):
        """TD_SYM vector of the given dictionary ids at width TD_SYM_W8..W64 (0..3)."""
        ids = np.asarray(ids)
        n = len(ids)
        p = self.check(self.lib.td_sym_vec_new(width, n), "sym_vec")
        C.cast(p + 24, C.POINTER(C.c_int64))[0] = n
        if n:
            dt = SYM_NP[width]
            buf = (C.c_char * (n * np.dtype(dt).itemsize)).from_address(p + 32)
            np.frombuffer(buf, dt, n)[:] = ids.astype(dt)
        return p

    def vec_alloc(self, typ, n):
        """New vector of n elements; returns (ptr, writable numpy view)."""
        p = self.check(self.lib.td_vec_new(typ, n), "vec_new")
        C.cast(p + 24, C.POINTER(C.c_int64))[0] = n
        return p, self.vec_view(p)

    def table(self, cols: dict) -> int:
        t = self.check(self.lib.td_table_new(len(cols)))
        for name, arr in cols.items():
            if isinstance(arr, int):
                v = arr
                self.lib.td_retain(v)
            elif isinstance(arr, tuple):
                v = self.vec(arr[0], arr[1])
            else:
                v = self.vec(arr)
            t = self.check(self.lib.td_table_add_col(t, self.sym(name), v))
            self.lib.td_release(v)
        return t

    def table_dict(self, t) -> dict:
        out = {}
        for j in range(self.lib.td_table_ncols(t)):
            col = self.lib.td_table_get_col_idx(t, j)
            out[self.sym_name(self.lib.td_table_col_name(t, j))] = self.to_numpy(col)
        return out

    def release(self, p):
        if p and p >= 32:
            self.lib.td_release(p)

    def graph(self, tbl=None) -> "Graph":
        return Graph(self, tbl)


class Graph:
    """DAG builder mirroring td.h's builder functions."""

    def __init__(self, td: Td, tbl=None):
        self.td = td
        self.L = td.lib
        self.g = self.L.td_graph_new(tbl or None)
        if not self.g:
            raise TdError(1, "graph")

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.free()

    def free(self):
        if self.g:
            self.L.td_graph_free(self.g)
            self.g = None

    def _ok(self, p, what):
        if not p:
            raise TdError(7, what)
        return p

    def scan(self, name):
        return self._ok(self.L.td_scan(self.g, name.encode()), "scan " + name)

    def scan_table(self, tid, name):
        return self._ok(self.L.td_scan_table(self.g, tid, name.encode()), "scan " + name)

    def add_table(self, t):
        return self.L.td_graph_add_table(self.g, t)

    def i64(self, v):
        return self._ok(self.L.td_const_i64(self.g, int(v)), "const")

    def f64(self, v):
        return self._ok(self.L.td_const_f64(self.g, float(v)), "const")

    def boolean(self, v):
        return self._ok(self.L.td_const_bool(self.g, bool(v)), "const")

    def string(self, s):
        return self._ok(self.L.td_const_str(self.g, s.encode()), "const")

    def const_table(self, t):
        return self._ok(self.L.td_const_table(self.g, t), "const table")

    def const_vec(self, v):
        return self._ok(self.L.td_const_vec(self.g, v), "const vec")

    def op(self, name, *args):
        return self._ok(getattr(self.L, "td_" + name)(self.g, *args), name)

    def filter(self, inp, pred):
        return self._ok(self.L.td_filter(self.g, inp, pred), "filter")

    def group(self, keys, ops, ins):
        nk, na = len(keys), len(ops)
        K = (P * max(nk, 1))(*keys)
        O = (C.c_uint16 * max(na, 1))(*ops)
        I = (P * max(na, 1))(*ins)
        return self._ok(self.L.td_group(self.g, K, nk, O, I, na), "group")

    def join(self, left, lkeys, right, rkeys, join_type=0):
        n = len(lkeys)
        LK = (P * n)(*lkeys)
        RK = (P * n)(*rkeys)
        return self._ok(self.L.td_join(self.g, left, LK, right, RK, n, join_type), "join")

    def sort(self, table_node, keys, descs=None, nulls_first=None):
        """td_sort_op: rows of table_node ordered by the key columns (scans);
        nulls_first None keeps Teide's default (DESC flags)."""
        n = len(keys)
        K = (P * max(n, 1))(*keys)
        D = (C.c_uint8 * max(n, 1))(*(descs or [0] * n))
        NF = (C.c_uint8 * max(n, 1))(*nulls_first) if nulls_first is not None else None
        return self._ok(self.L.td_sort_op(self.g, table_node, K, D, NF, n), "sort")

    def head(self, inp, n):
        return self._ok(self.L.td_head(self.g, inp, int(n)), "head")

    def execute(self, root, optimize=True):
        if optimize:
            root = self.L.td_optimize(self.g, root) or root
        return self.td.check(self.L.td_execute(self.g, root), "execute")
