"""tdg_group_run_static: the group-by entry point that allocates nothing.

It serves callers that cannot call cudaMalloc themselves (an engine embedded
in a process whose device memory is owned by another runtime's allocator, or
a latency-critical path that cannot take cudaMalloc's device-wide
synchronization): they pass inputs and outputs, and the scratch comes from a
16 MiB array compiled into the library.  The test calls it through the C ABI
twice in a row on different data -- so the second call would see anything the
first left behind -- and checks each result against tdg_group_run with a
caller-provided workspace: keys, counts and integer aggregates bit-exact, F64
aggregates within 1e-12 relative (atomic summation order differs between
runs).  The cases reach every plan that fits the array: shared-memory slots, global
records, the hash table, and the hot-slot sampling of inputs of 2^22 rows or
more.  It also checks that a group-by needing more scratch than the array
holds -- the partitioned method among them -- is refused with TD_ERR_RANGE.  The file sorts last so that a run
stopping at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

I64, F64 = 6, 7
OP_SUM, OP_MIN, OP_MAX, OP_COUNT, OP_AVG = 50, 52, 53, 54, 55
TD_ERR_RANGE = 3


def _bind():
    import teide_b200
    from teide_b200 import tdg as T
    t = teide_b200.device_abi()
    fn = t.lib.tdg_group_run_static
    fn.restype = C.c_int32
    fn.argtypes = [C.POINTER(T.GroupDesc), C.POINTER(T.Expr), C.c_void_p, C.POINTER(T.GroupOut), C.c_void_p]
    return t, T


def _desc(T, keys, key_lo, key_hi, v1, v2, v3=None):
    """SUM/MIN/MAX/COUNT of v1, AVG/SUM of v2 (F64), and SUM of v3 when given
    (a third distinct input column, which keeps the partitioned method out)."""
    d = T.GroupDesc()
    d.nrows = keys.numel()
    d.n_keys = 1
    d.keys[0] = T.col(keys.data_ptr(), I64)
    aggs = [(OP_SUM, v1, I64), (OP_MIN, v1, I64), (OP_MAX, v1, I64), (OP_COUNT, v1, I64), (OP_AVG, v2, F64),
            (OP_SUM, v2, F64)]
    if v3 is not None:
        aggs.append((OP_SUM, v3, I64))
    d.n_aggs = len(aggs)
    for a, (op, t, ty) in enumerate(aggs):
        d.aggs[a].op = op
        d.aggs[a].in_ = T.col(t.data_ptr(), ty)
    if key_lo is not None:
        d.have_range = 1
        d.key_min[0] = key_lo
        d.key_max[0] = key_hi
    return d


def _outputs(T, torch, plan, n_aggs):
    o = T.GroupOut()
    bufs = [torch.empty(max(plan.max_groups, 1), dtype=torch.int64, device="cuda")]
    o.keys[0] = bufs[0].data_ptr()
    for a in range(n_aggs):
        bufs.append(torch.empty(max(plan.max_groups, 1), dtype=torch.int64, device="cuda"))
        o.aggs[a] = bufs[-1].data_ptr()
    ng = torch.zeros(1, dtype=torch.int64, device="cuda")
    o.d_n_groups = ng.data_ptr()
    return o, bufs, ng


def _read(bufs, ng):
    n = int(ng.item())
    cols = [b[:n].cpu().numpy() for b in bufs]
    order = np.argsort(cols[0], kind="stable")
    return [c[order] for c in cols]


# direct_smem: every slot in shared memory; direct_global: global records;
# hash: the hash table; sampled: 4.2M rows (at least 2^22), so the hot-slot
# sampling tables are built and read -- with three distinct input columns,
# which keep the partitioned method (whose entry buffers alone need 12 bytes
# per row, more than the array holds at 2^20 rows) out of the plan.
CASES = {"direct_smem": (300_000, 64), "direct_global": (1_000_000, 5_000), "hash": (60_000, 20_000),
         "sampled": (4_200_000, 5_000)}


@pytest.mark.parametrize("case", list(CASES))
def test_static_group_matches_workspace_group(case):
    import torch
    t, T = _bind()
    torch.cuda.set_device(0)
    stream = torch.cuda.current_stream().cuda_stream
    n, k = CASES[case]
    for call in range(2):
        g = torch.Generator(device="cuda").manual_seed(100 * call + n)
        if case == "hash":
            universe = torch.randint(-2**62, 2**62, (k,), dtype=torch.int64, device="cuda", generator=g)
            keys = universe[torch.randint(0, k, (n,), device="cuda", generator=g)]
            lo = hi = None
        elif case == "sampled":
            # a skewed key set (half the rows on 40 keys), different on each call
            hot = torch.randint(0, k, (40,), dtype=torch.int64, device="cuda", generator=g)
            keys = torch.randint(0, k, (n,), dtype=torch.int64, device="cuda", generator=g)
            pick = torch.rand(n, device="cuda", generator=g) < 0.5
            keys = torch.where(pick, hot[torch.randint(0, 40, (n,), device="cuda", generator=g)], keys)
            lo, hi = 0, k - 1
        else:
            keys = torch.randint(0, k, (n,), dtype=torch.int64, device="cuda", generator=g)
            lo, hi = 0, k - 1
        v1 = torch.randint(-10**6, 10**6, (n,), dtype=torch.int64, device="cuda", generator=g)
        v2 = torch.randn(n, dtype=torch.float64, device="cuda", generator=g)
        v3 = torch.randint(-10**9, 10**9, (n,), dtype=torch.int64, device="cuda", generator=g) \
            if case == "sampled" else None
        d = _desc(T, keys, lo, hi, v1, v2, v3)
        plan = T.GroupPlan()
        assert t.tdg_group_plan_make(C.byref(d), 0, C.byref(plan)) == 0
        assert plan.ws_bytes <= 16 << 20
        ws = torch.empty(plan.ws_bytes, dtype=torch.uint8, device="cuda")
        oa, ba, na = _outputs(T, torch, plan, d.n_aggs)
        ob, bb, nb = _outputs(T, torch, plan, d.n_aggs)
        assert t.tdg_group_run(C.byref(d), None, None, C.byref(plan), ws.data_ptr(), C.byref(oa), stream) == 0
        assert t.lib.tdg_group_run_static(C.byref(d), None, None, C.byref(ob), stream) == 0
        torch.cuda.synchronize()
        ra, rb = _read(ba, na), _read(bb, nb)
        assert len(ra[0]) == len(rb[0]) > 0
        for i in range(len(ra)):
            if i in (5, 6):                      # AVG, SUM of F64 (bits as int64)
                fa, fb = ra[i].view(np.float64), rb[i].view(np.float64)
                assert np.allclose(fa, fb, rtol=1e-12, atol=1e-12), (case, call, i)
            else:                                # keys, integer aggregates, COUNT
                assert np.array_equal(ra[i], rb[i]), (case, call, i)


# records: 4M direct-array slots take more than 16 MiB; partitioned: 1.2M
# rows and 5000 slots plan the partitioned method, whose per-row entry
# buffers and sampling tables do not fit the array either
@pytest.mark.parametrize("n,k", [(1 << 22, 1 << 22), (1_200_000, 5_000)], ids=["records", "partitioned"])
def test_static_group_refuses_oversized_scratch(n, k):
    import torch
    t, T = _bind()
    torch.cuda.set_device(0)
    keys = torch.zeros(n, dtype=torch.int64, device="cuda")
    v1 = torch.zeros(n, dtype=torch.int64, device="cuda")
    v2 = torch.zeros(n, dtype=torch.float64, device="cuda")
    d = _desc(T, keys, 0, k - 1, v1, v2)
    plan = T.GroupPlan()
    assert t.tdg_group_plan_make(C.byref(d), 0, C.byref(plan)) == 0
    assert plan.ws_bytes > 16 << 20
    o, bufs, ng = _outputs(T, torch, plan, d.n_aggs)
    stream = torch.cuda.current_stream().cuda_stream
    assert t.lib.tdg_group_run_static(C.byref(d), None, None, C.byref(o), stream) == TD_ERR_RANGE
