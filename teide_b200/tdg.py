"""ctypes binding of the device-path C ABI (include/tdg.h).

The structs mirror tdg.h field for field.  Device buffers are passed as plain
integer addresses (e.g. torch.Tensor.data_ptr()); the stream as an integer
handle (torch.cuda.current_stream().cuda_stream) or 0.
"""
from __future__ import annotations

import ctypes as C

MAX_INS, MAX_XCOLS, MAX_KEYS, MAX_AGGS = 24, 8, 8, 8
GROUP_DIRECT, GROUP_HASH = 1, 2
JOIN_DIRECT, JOIN_HASH = 1, 2


class Col(C.Structure):
    _fields_ = [("data", C.c_void_p), ("type", C.c_int8), ("attrs", C.c_uint8), ("side", C.c_uint8),
                ("pad", C.c_uint8 * 5)]


class Ins(C.Structure):
    _fields_ = [("op", C.c_uint8), ("a", C.c_uint8), ("b", C.c_uint8), ("kind", C.c_uint8),
                ("pad", C.c_uint8 * 4), ("imm", C.c_int64)]


class Expr(C.Structure):
    _fields_ = [("n_ins", C.c_int32), ("n_cols", C.c_int32), ("out", C.c_int32), ("pad", C.c_int32),
                ("cols", Col * MAX_XCOLS), ("ins", Ins * MAX_INS)]


class Agg(C.Structure):
    _fields_ = [("op", C.c_int32), ("pad", C.c_int32), ("in_", Col)]


class GroupDesc(C.Structure):
    _fields_ = [("nrows", C.c_int64), ("n_keys", C.c_int32), ("n_aggs", C.c_int32),
                ("keys", Col * MAX_KEYS), ("aggs", Agg * MAX_AGGS), ("have_range", C.c_int32),
                ("pad", C.c_int32), ("key_min", C.c_int64 * MAX_KEYS), ("key_max", C.c_int64 * MAX_KEYS)]


class GroupPlan(C.Structure):
    _fields_ = [("method", C.c_int32), ("smem", C.c_int32), ("n_slots", C.c_int64),
                ("max_groups", C.c_int64), ("ws_bytes", C.c_size_t), ("ctas_per_sm", C.c_int32),
                ("pad", C.c_int32)]


class GroupOut(C.Structure):
    _fields_ = [("keys", C.c_void_p * MAX_KEYS), ("aggs", C.c_void_p * MAX_AGGS),
                ("d_n_groups", C.c_void_p)]


class JoinDesc(C.Structure):
    _fields_ = [("n_left", C.c_int64), ("n_right", C.c_int64), ("n_keys", C.c_int32),
                ("join_type", C.c_int32), ("lkeys", Col * MAX_KEYS), ("rkeys", Col * MAX_KEYS),
                ("have_range", C.c_int32), ("flags", C.c_int32), ("rkey_min", C.c_int64),
                ("rkey_max", C.c_int64)]


class JoinPlan(C.Structure):
    _fields_ = [("method", C.c_int32), ("pad", C.c_int32), ("n_slots", C.c_int64), ("ws_bytes", C.c_size_t)]


def col(ptr, typ, attrs=0, side=0):
    c = Col()
    c.data = ptr
    c.type = typ
    c.attrs = attrs
    c.side = side
    return c


class Tdg:
    """Typed entry points of tdg.h on a loaded library (ctypes.CDLL)."""

    def __init__(self, lib):
        self.lib = lib
        P = C.c_void_p
        sig = {
            "tdg_minmax": (C.c_int32, [Col, C.c_int64, P, P]),
            "tdg_group_plan_make": (C.c_int32, [C.POINTER(GroupDesc), C.c_int64, C.POINTER(GroupPlan)]),
            "tdg_group_run": (C.c_int32, [C.POINTER(GroupDesc), C.POINTER(Expr), P, C.POINTER(GroupPlan),
                                          P, C.POINTER(GroupOut), P]),
            "tdg_join_plan_make": (C.c_int32, [C.POINTER(JoinDesc), C.POINTER(JoinPlan)]),
            "tdg_join_build": (C.c_int32, [C.POINTER(JoinDesc), C.POINTER(JoinPlan), P, P]),
            "tdg_join_group_run": (C.c_int32, [C.POINTER(JoinDesc), C.POINTER(JoinPlan), P, C.POINTER(Expr), P,
                                               C.POINTER(GroupDesc), C.POINTER(GroupPlan), P,
                                               C.POINTER(GroupOut), P]),
            "tdg_select_ws_bytes": (C.c_size_t, [C.c_int64]),
            "tdg_set_timing": (None, [C.c_int32]),
            "tdg_last_main_ms": (C.c_float, []),
            "tdg_last_build_ms": (C.c_float, []),
            "tdg_launch_count": (C.c_uint64, []),
            "tdg_device_sm_count": (C.c_int32, []),
        }
        for name, (res, args) in sig.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args

    def __getattr__(self, name):
        return getattr(self.lib, name)
