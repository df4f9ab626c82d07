"""td_server queue logic on the host: FIFO admission, the memory budget and
the queue capacity.  Without a GPU every execution fails fast with
TD_ERR_IO, which still drives the request loop end to end."""
import numpy as np
import pytest

import teide_b200
from teide_b200 import serve
from teide_b200.td import OP_SUM, TdError

TD_ERR_IO, TD_ERR_RANGE = 8, 3


@pytest.fixture(scope="module")
def td():
    t = teide_b200.load()
    if t.lib.td_gpu_device_count() > 0:
        pytest.skip("host-only test: a GPU would make the executions succeed")
    return t


def _graphs(td, n):
    tbl = td.table({"k": np.arange(100, dtype=np.int64) % 7, "v": np.arange(100, dtype=np.int64)})
    gs = []
    for _ in range(n):
        g = td.graph(tbl)
        gs.append((g, g.group([g.scan("k")], [OP_SUM], [g.scan("v")])))
    return tbl, gs


def test_fifo_admission_and_status(td):
    tbl, gs = _graphs(td, 40)
    with serve.Server(td, slots=4, hbm_budget=1 << 40) as s:
        ts = [s.submit(g, r) for g, r in gs]
        starts = []
        for t in ts:
            res, tm = s.wait(t)
            assert res == TD_ERR_IO and tm.status == TD_ERR_IO
            assert tm.submit_ns <= tm.start_ns <= tm.end_ns
            starts.append(tm.start_ns)
        assert starts == sorted(starts)            # admitted in arrival order
        st = s.stats()
        assert st.completed == 40 and st.queued == 0 and st.in_flight == 0 and st.reserved_bytes == 0
        assert 1 <= st.peak_in_flight <= 4
    for g, _ in gs:
        g.free()
    td.release(tbl)


def test_budget_admits_one_at_a_time(td):
    tbl, gs = _graphs(td, 16)
    with serve.Server(td, slots=8, hbm_budget=1) as s:   # every estimate exceeds 1 byte
        ts = [s.submit(g, r, est_bytes=1 << 20) for g, r in gs]
        for t in ts:
            s.wait(t)
        st = s.stats()
        assert st.peak_in_flight == 1                     # oversized requests run alone
        assert st.peak_reserved_bytes == 1 << 20
    for g, _ in gs:
        g.free()
    td.release(tbl)


def test_queue_capacity_and_bad_ticket(td):
    tbl, gs = _graphs(td, 5)
    with serve.Server(td, slots=2, queue_cap=4) as s:
        ts = [s.submit(g, r) for g, r in gs[:4]]
        with pytest.raises(TdError) as e:               # 4 results not yet collected
            s.submit(*gs[4])
        assert e.value.code == TD_ERR_RANGE
        for t in ts:
            s.wait(t)
        t5 = s.submit(*gs[4])                           # slots free again
        s.wait(t5)
        res, _ = s.wait(t5)                             # collected already
        assert res == TD_ERR_RANGE
    for g, _ in gs:
        g.free()
    td.release(tbl)


def test_estimate_counts_uploads(td):
    tbl, gs = _graphs(td, 1)
    g, root = gs[0]
    est = td.lib.td_server_estimate(g.g, root)
    assert est >= 100 * 16 + 100 * 128                  # both columns uploaded + scratch bound
    g.free()
    td.release(tbl)
