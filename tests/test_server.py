"""The request loop (gx_server_*) on the CPU, with an executor that only
sleeps: admission earliest deadline first (arrival order without deadlines),
one request per job on the GPU at a
time, the HBM budget (resident jobs + what requests in flight add), the slot
count, rejection of what can never fit, and the latency statistics."""
import threading
import time

import pytest

from difx_b200 import capi, gxcorr


def _sd(i):
    return capi.SubintDesc(0, 0, i, 0.0, [], [], [], 0)


class Recorder:
    def __init__(self, dur=0.04):
        self.dur = dur
        self.lock = threading.Lock()
        self.events = []   # (job, start, end, tag)

    def __call__(self, job, sub, res):
        t0 = time.monotonic()
        time.sleep(self.dur)
        with self.lock:
            self.events.append((job, t0, time.monotonic(), res))
        return 0


def _max_overlap(ev, pred=lambda e: True):
    pts = []
    for e in ev:
        if pred(e):
            pts += [(e[1], 1), (e[2], -1)]
    pts.sort(key=lambda p: (p[0], p[1]))
    cur = best = 0
    for _, d in pts:
        cur += d
        best = max(best, cur)
    return best


def test_jobs_exclusive_slots_and_budget():
    srv = gxcorr.Server(slots=4, hbm_budget_bytes=1000)
    rec = Recorder()
    srv.set_executor(rec)
    jobs = [srv.attach(None, r) for r in (100, 200, 300)]          # 600 resident, 400 left
    tickets = []
    for k in range(12):
        j = jobs[k % 3] if k < 9 else jobs[0]
        tickets.append(srv.submit(j, _sd(k), results_ptr=k + 1, request_bytes=150))
    lat = [srv.wait(t) for t in tickets]
    st = srv.stats()
    srv.close()
    assert st.completed == 12 and st.failed == 0
    assert len(rec.events) == 12
    # one request per job on the GPU at a time
    for j in jobs:
        assert _max_overlap(rec.events, lambda e, j=j: e[0] == j) == 1
    # 400 bytes left for requests of 150: at most two in flight, although 4 slots exist
    assert _max_overlap(rec.events) == 2
    assert all(x >= rec.dur * 1000 * 0.9 for x in lat)
    assert st.p50_ms <= st.p95_ms <= st.p99_ms <= st.max_ms


def test_arrival_order_with_one_slot():
    srv = gxcorr.Server(slots=1, hbm_budget_bytes=1 << 20)
    rec = Recorder(0.01)
    srv.set_executor(rec)
    a, b = srv.attach(None, 0), srv.attach(None, 0)
    tickets = [srv.submit(a if k % 2 else b, _sd(k), results_ptr=k + 1, request_bytes=0) for k in range(8)]
    for t in tickets:
        srv.wait(t)
    srv.close()
    assert [e[3] for e in rec.events] == list(range(1, 9))


def test_requests_overlap_across_jobs():
    srv = gxcorr.Server(slots=3, hbm_budget_bytes=1 << 20)
    rec = Recorder(0.1)
    srv.set_executor(rec)
    jobs = [srv.attach(None, 10) for _ in range(3)]
    t0 = time.monotonic()
    tickets = [srv.submit(j, _sd(i), results_ptr=i + 1, request_bytes=0) for i, j in enumerate(jobs)]
    for t in tickets:
        srv.wait(t)
    wall = time.monotonic() - t0
    srv.close()
    assert _max_overlap(rec.events) == 3
    assert wall < 0.25   # three 0.1 s requests ran together


def test_what_never_fits_is_refused():
    srv = gxcorr.Server(slots=2, hbm_budget_bytes=1000)
    srv.set_executor(Recorder(0.0))
    j = srv.attach(None, 900)
    with pytest.raises(gxcorr.GxError) as e:
        srv.attach(None, 200)
    assert e.value.status == 4   # GX_ERR_NOMEM
    with pytest.raises(gxcorr.GxError) as e:
        srv.submit(j, _sd(0), request_bytes=101)
    assert e.value.status == 4
    t = srv.submit(j, _sd(1), request_bytes=100)
    srv.wait(t)
    srv.close()


def test_earliest_deadline_first():
    """With one slot busy, queued requests start in order of their deadlines
    (submission + the job's relative deadline), not of their arrival; jobs
    without a deadline come after those with one, in arrival order."""
    srv = gxcorr.Server(slots=1, hbm_budget_bytes=1 << 20)
    rec = Recorder(0.03)
    srv.set_executor(rec)
    slow, urgent, loose, none = (srv.attach(None, 0) for _ in range(4))
    srv.set_deadline(slow, 1000.0)
    srv.set_deadline(urgent, 50.0)
    srv.set_deadline(loose, 500.0)
    t = [srv.submit(slow, _sd(0), results_ptr=1, request_bytes=0)]   # occupies the slot
    time.sleep(0.01)
    t.append(srv.submit(none, _sd(1), results_ptr=2, request_bytes=0))
    t.append(srv.submit(loose, _sd(2), results_ptr=3, request_bytes=0))
    t.append(srv.submit(slow, _sd(3), results_ptr=4, request_bytes=0))
    t.append(srv.submit(urgent, _sd(4), results_ptr=5, request_bytes=0))
    for x in t:
        srv.wait(x)
    srv.close()
    assert [e[3] for e in rec.events] == [1, 5, 3, 4, 2]
