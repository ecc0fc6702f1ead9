"""CPU: the request server's failure handling (deadlines, cancellation, a
stuck slot) with host-only stand-in slots -- no device work, nothing that
could fault or hang a GPU.  A stand-in "kernel" polls its slot's abort flag
the way the library's persistent kernels poll pcf_ctx_abort's word, and
raises the library's timeout error when it sees it; a "hung" one ignores it,
which is what the stuck-slot watchdog is for."""
import threading
import time

import numpy as np
import pytest

from desi_b200._lib import PCF_ERR_TIMEOUT, PcfError
from desi_b200.serve import DeadlineExceeded, PcfServer, Request, RequestCancelled, SlotStuck


class FakeSlot:
    def __init__(self, server, idx):
        self.idx = idx
        self.current = None
        self.aborted = False
        self.retired = False
        self._abort = threading.Event()
        self._never = threading.Event()
        self.runs = 0

    def abort(self, on=True):
        if on:
            self._abort.set()
        else:
            self._abort.clear()

    def run(self, req):
        self.runs += 1
        if req.kind == "hang":  # ignores the abort request
            self._never.wait(30.0)
            return {"_units": 0.0}
        if req.kind == "slow":  # polls the abort flag, like the kernels
            t_end = time.perf_counter() + 10.0
            while time.perf_counter() < t_end:
                if self._abort.is_set():
                    raise PcfError(PCF_ERR_TIMEOUT, "fake kernel", "abort requested")
                time.sleep(0.001)
        return {"_units": 1.0, "rid": req.rid}


def _server(slots=2, **kw):
    srv = PcfServer(slots=slots, hbm_budget=1 << 40, slot_factory=FakeSlot, **kw)
    srv.catalogs = {"c": {"points": np.zeros((100, 4), np.float32), "box": 100.0}}
    return srv


def _req(kind, rid, deadline=None):
    return Request(kind, "c", "c", 10, 10.0, rid=rid, deadline_s=deadline)


def test_deadline_aborts_a_running_request_and_the_slot_serves_on():
    srv = _server(slots=1)
    try:
        slow = _req("slow", 1, deadline=0.1)
        t0 = time.perf_counter()
        srv.submit(slow)
        with pytest.raises(DeadlineExceeded):
            slow.future.result(timeout=5)
        assert time.perf_counter() - t0 < 2.0
        ok = _req("fast", 2)
        assert srv.submit(ok).result(timeout=5)["rid"] == 2
        assert not srv.slots[0]._abort.is_set()  # cleared before the next call
    finally:
        srv.close()


def test_deadline_drops_a_pending_request():
    srv = _server(slots=1)
    try:
        blocker = _req("slow", 1)
        srv.submit(blocker)
        time.sleep(0.05)
        late = _req("fast", 2, deadline=0.05)
        srv.submit(late)
        with pytest.raises(DeadlineExceeded):
            late.future.result(timeout=5)
        assert srv.cancel(blocker)
        with pytest.raises(RequestCancelled):
            blocker.future.result(timeout=5)
    finally:
        srv.close()


def test_cancel_pending_and_running():
    srv = _server(slots=1)
    try:
        running = _req("slow", 1)
        pending = _req("fast", 2)
        srv.submit(running)
        time.sleep(0.05)
        srv.submit(pending)
        assert srv.cancel(pending)
        with pytest.raises(RequestCancelled):
            pending.future.result(timeout=5)
        t0 = time.perf_counter()
        assert srv.cancel(running)
        with pytest.raises(RequestCancelled):
            running.future.result(timeout=5)
        assert time.perf_counter() - t0 < 2.0
        done = _req("fast", 3)
        srv.submit(done).result(timeout=5)
        assert not srv.cancel(done)  # already complete
    finally:
        srv.close()


def test_stuck_slot_is_retired_and_the_others_serve_on():
    srv = _server(slots=2, stuck_after_s=0.1, stuck_grace_s=0.2)
    try:
        hung = _req("hang", 1)
        srv.submit(hung)
        time.sleep(0.05)
        with pytest.raises(SlotStuck):
            hung.future.result(timeout=5)
        stuck = [s for s in srv.slots if s.retired]
        assert len(stuck) == 1 and stuck[0]._abort.is_set()
        # the other slot keeps serving; the retired one takes nothing more
        outs = [srv.submit(_req("fast", 10 + i)) for i in range(5)]
        assert [f.result(timeout=5)["rid"] for f in outs] == [10, 11, 12, 13, 14]
        assert stuck[0].runs == 1
    finally:
        for s in srv.slots:
            s._never.set()
        srv.close()


def test_slow_request_within_the_stuck_limit_is_not_touched():
    srv = _server(slots=1, stuck_after_s=5.0)
    try:
        f = srv.submit(_req("fast", 1))
        assert f.result(timeout=5)["rid"] == 1
        assert not srv.slots[0].retired
    finally:
        srv.close()
