"""Admission core of the reconstruction server (CPU, no GPU): requests run
only while their footprint fits into free memory minus the reserve and the
running requests; small requests pass a large one that does not fit; an
idle device always takes the queue head; failures stay on their request."""
import threading
import time

import numpy as np

from monalisa_b200.serving import ReconRequest, Scheduler, latency_stats


class Req(ReconRequest):
    def __init__(self, rid, nbytes, dur=0.05, fail=False):
        super().__init__(t=None, ve=None, C=None, y=None, N_u=None, n_u=None, rid=rid)
        self.nbytes, self.dur, self.fail = nbytes, dur, fail

    def device_bytes(self):
        return self.nbytes


def _server(free, workers=4):
    state = {"running": 0, "bytes": 0, "peak_bytes": 0}
    lock = threading.Lock()

    def execute(req, worker):
        with lock:
            state["running"] += 1
            state["bytes"] += req.nbytes
            state["peak_bytes"] = max(state["peak_bytes"], state["bytes"])
        time.sleep(req.dur)
        with lock:
            state["running"] -= 1
            state["bytes"] -= req.nbytes
        if req.fail:
            raise RuntimeError("planted failure")
        return np.full(1, req.rid)

    return Scheduler(execute, lambda: free, workers=workers, reserve_bytes=10), state


def test_memory_admission_and_bypass():
    sched, state = _server(free=110, workers=4)
    big = [Req(i, 60, 0.1) for i in range(3)]
    small = [Req(10 + i, 20, 0.02) for i in range(4)]
    reqs = [sched.submit(r) for r in (big[0], big[1], small[0], small[1], big[2], small[2], small[3])]
    for r in reqs:
        assert r.done.wait(10)
    sched.close()
    assert state["peak_bytes"] <= 100  # free - reserve
    order = sched.order
    # big[1] cannot start beside big[0]; the small requests behind it pass it
    assert order.index(10) < order.index(1) and order.index(11) < order.index(1)
    assert all(r.x is not None and r.x[0] == r.rid for r in reqs)
    st = latency_stats(reqs)
    assert st["n"] == 7 and st["errors"] == 0 and st["p99_ms"] >= st["p50_ms"] > 0


def test_idle_device_takes_an_oversized_head_and_failures_stay_local():
    sched, _ = _server(free=50, workers=2)
    huge = sched.submit(Req(1, 500, 0.02))        # larger than the whole budget
    bad = sched.submit(Req(2, 10, 0.01, fail=True))
    ok = sched.submit(Req(3, 10, 0.01))
    for r in (huge, bad, ok):
        assert r.done.wait(10)
    sched.close()
    assert huge.error is None and huge.x[0] == 1
    assert bad.error and "planted failure" in bad.error and bad.x is None
    assert ok.error is None and ok.x[0] == 3


def test_footprint_estimate_grows_with_the_problem():
    def req(n, N, nPt, nCh):
        t = np.zeros((3, nPt))
        return ReconRequest(t=t, ve=np.ones(nPt), C=np.ones((n ** 3, nCh)), y=None, N_u=np.array([N] * 3),
                            n_u=np.array([n] * 3))

    small, big = req(96, 192, 256_000, 8), req(128, 256, 1_048_576, 16)
    assert 0 < small.device_bytes() < big.device_bytes()
    # the c2-size request needs a few GB, far below one B200's memory
    assert 2e9 < big.device_bytes() < 2e10
