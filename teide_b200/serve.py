"""Serving: submit td.h graphs to the GPU request loop (td_server, td_b200.h).

The server runs `slots` queries at once, each on its own CUDA stream, and
admits waiting queries in arrival order as slots and device memory free up.
This module binds it and builds the two request shapes of the served mix:

  group  README-style filter + group-by over a contiguous row range of a
         resident table (the range is a zero-copy slice view);
  join   filter over a row range of a resident probe table, inner join to a
         resident build table, group-by -- one fused graph.
"""
import ctypes as C
import time

import numpy as np

from .td import OP_AVG, OP_COUNT, OP_MAX, OP_MIN, OP_SUM, P, TdError


class Timing(C.Structure):
    _fields_ = [("submit_ns", C.c_int64), ("start_ns", C.c_int64), ("end_ns", C.c_int64),
                ("est_bytes", C.c_int64), ("status", C.c_int32), ("in_flight_at_start", C.c_int32)]


class Stats(C.Structure):
    _fields_ = [("completed", C.c_uint64), ("queued", C.c_int64), ("in_flight", C.c_int32),
                ("peak_in_flight", C.c_int32), ("slots", C.c_int32), ("pad", C.c_int32),
                ("budget_bytes", C.c_uint64), ("reserved_bytes", C.c_uint64),
                ("peak_reserved_bytes", C.c_uint64)]


def _bind(L):
    if getattr(L, "_td_server_bound", False):
        return
    L.td_server_new.restype = P
    L.td_server_new.argtypes = [C.c_int32, C.c_size_t, C.c_int64]
    L.td_server_submit.restype = C.c_int64
    L.td_server_submit.argtypes = [P, P, P, C.c_size_t]
    L.td_server_wait.restype = P
    L.td_server_wait.argtypes = [P, C.c_int64, C.POINTER(Timing)]
    L.td_server_stats.restype = None
    L.td_server_stats.argtypes = [P, C.POINTER(Stats)]
    L.td_server_free.restype = None
    L.td_server_free.argtypes = [P]
    L.td_server_estimate.restype = C.c_size_t
    L.td_server_estimate.argtypes = [P, P]
    L.td_vec_slice.restype = P
    L.td_vec_slice.argtypes = [P, C.c_int64, C.c_int64]
    L._td_server_bound = True


class Server:
    def __init__(self, td, slots=8, hbm_budget=0, queue_cap=0):
        self.td = td
        self.L = td.lib
        _bind(self.L)
        self.s = self.L.td_server_new(slots, hbm_budget, queue_cap)
        if not self.s:
            raise TdError(1, "td_server_new")

    def submit(self, graph, root, est_bytes=0):
        t = self.L.td_server_submit(self.s, graph.g, root, est_bytes)
        if t < 0:
            raise TdError(-t, "td_server_submit")
        return t

    def wait(self, ticket):
        """(result pointer or error code, Timing)."""
        tm = Timing()
        r = self.L.td_server_wait(self.s, ticket, C.byref(tm)) or 0
        return r, tm

    def stats(self):
        st = Stats()
        self.L.td_server_stats(self.s, C.byref(st))
        return st

    def close(self):
        if self.s:
            self.L.td_server_free(self.s)
            self.s = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def table_slice(td, tbl, off, n):
    """A table whose columns are zero-copy views of rows [off, off + n) of tbl."""
    _bind(td.lib)
    L = td.lib
    out = td.check(L.td_table_new(L.td_table_ncols(tbl)))
    for j in range(L.td_table_ncols(tbl)):
        col = L.td_table_get_col_idx(tbl, j)
        v = td.check(L.td_vec_slice(col, off, n), "td_vec_slice")
        out = td.check(L.td_table_add_col(out, L.td_table_col_name(tbl, j), v))
        L.td_release(v)
    return out


def _const(g, k):
    return g.f64(k) if isinstance(k, float) else g.i64(k)


GROUP_AGGS = [(OP_COUNT, "v1"), (OP_SUM, "v1"), (OP_MIN, "v1"), (OP_MAX, "v1"), (OP_AVG, "v2")]
JOIN_AGGS = [(OP_SUM, "price"), (OP_COUNT, "price")]


def group_request(td, tbl, threshold):
    """README form: group keys and aggregate inputs are filter(scan, v1 > t)."""
    g = td.graph(tbl)
    p = g.op("gt", g.scan("v1"), g.i64(int(threshold)))
    ks = [g.filter(g.scan("key"), p)]
    ins = [g.filter(g.scan(n), p) for _, n in GROUP_AGGS]
    root = g.group(ks, [a for a, _ in GROUP_AGGS], ins)
    return g, root


def join_request(td, build_t, probe_t, threshold):
    """group(cat; SUM(price), COUNT) over join(filter(probe, qty > t), build)."""
    g = td.graph(None)
    left = g.filter(g.const_table(probe_t), g.op("gt", g.scan("qty"), g.i64(int(threshold))))
    g.join(left, [g.scan("fk")], g.const_table(build_t), [g.scan("pk")], 0)
    root = g.group([g.scan("cat")], [a for a, _ in JOIN_AGGS], [g.scan(n) for _, n in JOIN_AGGS])
    return g, root


class Request:
    __slots__ = ("kind", "off", "n", "threshold", "arrival", "tbl", "graph", "root")

    def __init__(self, kind, off, n, threshold, arrival):
        self.kind, self.off, self.n, self.threshold, self.arrival = kind, off, n, threshold, arrival
        self.tbl = self.graph = self.root = None


def build(td, reqs, group_tbl, build_t, probe_t):
    """Give every request its range view and its graph (prepared queries)."""
    for r in reqs:
        if r.kind == "group":
            r.tbl = table_slice(td, group_tbl, r.off, r.n)
            r.graph, r.root = group_request(td, r.tbl, r.threshold)
        else:
            r.tbl = table_slice(td, probe_t, r.off, r.n)
            r.graph, r.root = join_request(td, build_t, r.tbl, r.threshold)


def release(td, reqs):
    for r in reqs:
        if r.graph:
            r.graph.free()
        td.release(r.tbl)
        r.graph = r.tbl = r.root = None


def run_open_loop(server, reqs, keep=None):
    """Submit each request at its arrival time (seconds after start) while a
    second thread waits for the results in order and releases them, as a
    client consuming answers would (results never pile up on the host).
    Returns (latencies_s, makespan_s, results) where results holds the result
    pointers of the indices in `keep` (others are released)."""
    import threading
    td = server.td
    keep = set(keep or ())
    tickets = [None] * len(reqs)
    ready = threading.Semaphore(0)
    lat, ends, results, errors = [0.0] * len(reqs), [0] * len(reqs), {}, []
    t0 = time.monotonic()
    start_ns = int(t0 * 1e9)

    def consume():
        for i, r in enumerate(reqs):
            ready.acquire()
            res, tm = server.wait(tickets[i])
            if tm.status:
                errors.append(TdError(tm.status, f"request {i} ({r.kind})"))
                continue
            arrival_ns = start_ns + int(r.arrival * 1e9)
            lat[i] = (tm.end_ns - min(arrival_ns, tm.submit_ns)) / 1e9
            ends[i] = tm.end_ns
            if i in keep:
                results[i] = res
            else:
                td.release(res)

    waiter = threading.Thread(target=consume, daemon=True)
    waiter.start()
    for i, r in enumerate(reqs):
        delay = t0 + r.arrival - time.monotonic()
        if delay > 0:
            time.sleep(delay)          # sleeps, never spins: the consumer needs the interpreter too
        tickets[i] = server.submit(r.graph, r.root)
        ready.release()
    waiter.join()
    if errors:
        raise errors[0]
    makespan = (max(ends) - start_ns) / 1e9 if ends else 0.0
    return np.array(lat), makespan, results


def run_closed(server, reqs):
    """Every request submitted at once (a second thread consumes the results
    in order as they complete); returns seconds until the last finished."""
    import threading
    td = server.td
    t0 = time.monotonic_ns()
    tickets = []
    ready = threading.Semaphore(0)
    end, errors = [t0], []

    def consume():
        for i in range(len(reqs)):
            ready.acquire()
            res, tm = server.wait(tickets[i])
            if tm.status:
                errors.append(TdError(tm.status, f"request {i}"))
                continue
            td.release(res)
            end[0] = max(end[0], tm.end_ns)

    waiter = threading.Thread(target=consume, daemon=True)
    waiter.start()
    for r in reqs:
        tickets.append(server.submit(r.graph, r.root))
        ready.release()
    waiter.join()
    if errors:
        raise errors[0]
    return (end[0] - t0) / 1e9
