"""CPU: the request server's scheduling (no device work): pending requests
go smallest expected work first, with an age bound."""
import collections
import threading
import time

import numpy as np


def test_shortest_expected_work_first_with_age_bound():
    """Pending requests go smallest expected work first; one that has waited
    past max_wait_s goes first regardless (host logic only, no launch)."""
    from desi_b200.serve import PcfServer, Request, request_work
    srv = PcfServer.__new__(PcfServer)  # scheduler state only: no slots, no device
    srv._lock = threading.Condition()
    srv._pending = collections.deque()
    srv._in_use = 0
    srv.hbm_budget = 1 << 40
    srv.max_wait_s = 10.0
    srv.catalogs = {"big": {"points": np.zeros((20000, 4), np.float32), "box": 500.0},
                    "small": {"points": np.zeros((500, 4), np.float32), "box": 500.0}}
    now = time.perf_counter()
    a = Request("2iso", "big", "big", 30, 80.0, rid=0)
    b = Request("2ani", "small", "small", 30, 80.0, rid=1)
    c = Request("3iso", "small", "small", 10, 40.0, rid=2)
    for r in (a, b, c):
        r.t_submit = now
        srv._pending.append(r)
    sizes = {k: len(v["points"]) for k, v in srv.catalogs.items()}
    boxes = {k: v["box"] for k, v in srv.catalogs.items()}
    order = sorted((a, b, c), key=lambda r: request_work(r, sizes, boxes))
    assert [srv._pick().rid for _ in range(3)] == [r.rid for r in order]
    # an old request jumps the queue
    a.t_submit, b.t_submit = now - 20.0, now
    srv._pending.extend([b, a])
    assert srv._pick() is a and srv._pick() is b
