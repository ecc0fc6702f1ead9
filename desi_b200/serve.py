"""Continuous-batching request server for correlation-function histograms.

Requests (2iso / 2ani / 3iso, optionally periodic) name catalogs registered
with the server.  The server keeps ``slots`` workers, each with its own
library context (its own CUDA stream and memory pool) and its own cache of
gridded catalogs resident in HBM (LRU by bytes).  A request is admitted as
soon as a slot is free *and* its HBM footprint fits the budget -- requests
that arrive while others run start immediately on another slot, so their
kernels overlap on the device (continuous batching, not a queue).  When
several requests wait, a free slot takes the one with the least expected
work (in-range pairs at uniform density), unless one has waited longer than
``max_wait_s``.  The library calls release the GIL (ctypes), so slots run
concurrently.

Failure handling (no device fault involved): a request may carry a
deadline and may be cancelled; a watchdog thread drops pending requests past
their deadline and, for a running one, asks its slot's context to abort
(pcf_ctx_abort: the persistent kernels stop at their next work item and the
call returns PCF_ERR_TIMEOUT), then fails the request's future with
DeadlineExceeded or RequestCancelled.  A slot whose request outlives
``stuck_after_s`` is aborted the same way; if it still has not returned
after a grace period, the slot is retired (its request fails with
SlotStuck) and the other slots keep serving.

Every result is computed by the same kernels whether a request runs alone
or in the mix; ``tests/test_serve.py`` checks that the histograms are
identical both ways.  ``python -m desi_b200.serve`` runs a seeded stream of
mixed requests with Poisson arrivals and prints latency p50/p99 and
throughput as one JSON line.
"""
from __future__ import annotations

import collections
import json
import math
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np

from . import _lib, api

KINDS = ("2iso", "2ani", "3iso")


class RequestCancelled(Exception):
    """The request was cancelled (PcfServer.cancel) before it completed."""


class DeadlineExceeded(Exception):
    """The request did not complete within its deadline."""


class SlotStuck(Exception):
    """The slot running the request stopped responding and was retired."""


@dataclass
class Request:
    kind: str
    data: str
    rand: str
    bins: int
    dmax: float
    bpc: bool = False
    arrival: float = 0.0  # seconds from stream start (run_stream)
    rid: int = 0
    deadline_s: float | None = None  # from submission; None: no deadline
    future: Future = field(default_factory=Future, repr=False)
    t_submit: float = 0.0
    t_start: float = 0.0
    t_end: float = 0.0
    slot: int = -1
    # why the request is being stopped (an exception class), set under the
    # server lock by cancel() or the watchdog
    stop_reason: type | None = field(default=None, repr=False)


def grid_bytes(n: int, partitions: int = 64) -> int:
    """Device bytes of one gridded catalog: raw copy, cell-ordered SoA planes,
    pair-packed copy and integer weights, cell table and tiles (upper bound),
    with each buffer rounded up to the library pool's size class (at most a
    quarter more)."""
    return (n * (16 + 16 + 16) + 4 * (partitions ** 3 + 1) + 16 * n) * 5 // 4 + (1 << 20)


def request_work(req: Request, sizes: dict, boxes: dict) -> float:
    """Expected candidate work of a request (its scheduling cost): in-range
    pairs of DD + RR + DR at uniform density, times the expected neighbours
    of a point for 3iso (triangles per pair)."""
    nd, nr = sizes[req.data], sizes[req.rand]
    box = boxes[req.data]
    frac = (2.0 if req.kind == "2ani" else 4.0 / 3.0) * math.pi * req.dmax ** 3 / box ** 3
    pairs = 0.5 * (nd * nd + nr * nr) * frac + nd * nr * frac
    if req.kind == "3iso":
        pairs *= max(nd, nr) * 4.0 / 3.0 * math.pi * req.dmax ** 3 / box ** 3
    return pairs


def request_bytes(req: Request, sizes: dict) -> int:
    """HBM footprint of a running request: its two grids (if it has to build
    them), histograms and scratch (triplet lists spill to per-SM scratch in
    the worst case)."""
    nb = req.bins ** (3 if req.kind == "3iso" else (2 if req.kind == "2ani" else 1))
    fp = 3 * 24 * nb + (8 << 20) + grid_bytes(sizes[req.data]) + grid_bytes(sizes[req.rand])
    if req.kind == "3iso":
        fp += 2 * 148 * 16 * max(sizes[req.data], sizes[req.rand])
    return fp


class _Slot:
    def __init__(self, server: "PcfServer", idx: int, device: int, cache_bytes: int):
        self.server = server
        self.idx = idx
        self.ctx = api.Context(device)
        self.cache = collections.OrderedDict()  # (catalog, box) -> (Grid, bytes)
        self.cache_bytes = cache_bytes
        self.used = 0
        self.busy = False
        self.current: Request | None = None  # the running request
        self.aborted = False                 # abort requested for the current request
        self.retired = False                 # declared stuck: takes no more requests

    def abort(self, on: bool = True) -> None:
        self.ctx.abort(on)

    def grid(self, name: str, keep=()) -> api.Grid:
        """The catalog gridded on this slot's device, built on first use and
        kept resident; least recently used grids (not in `keep`) are freed
        when the slot's cache exceeds its byte budget."""
        cat = self.server.catalogs[name]
        key = (name, cat["box"])
        if key in self.cache:
            self.cache.move_to_end(key)
            return self.cache[key][0]
        g = self.ctx.grid(cat["points"], cat["box"])
        b = grid_bytes(len(cat["points"]))
        self.cache[key] = (g, b)
        self.used += b
        for k in list(self.cache.keys()):
            if self.used <= self.cache_bytes:
                break
            if k == key or k[0] in keep:
                continue
            old, ob = self.cache.pop(k)
            old.free()
            self.used -= ob
        return g

    def run(self, req: Request) -> dict:
        keep = (req.data, req.rand)
        gd, gr = self.grid(req.data, keep), self.grid(req.rand, keep)
        c = self.ctx
        if req.kind == "3iso":
            kw = dict(bins=req.bins, dmax=req.dmax, bpc=req.bpc, stats=True)
            out, tri = {}, 0.0
            for name, x, y in (("DDD", gd, None), ("RRR", gr, None), ("DDR", gd, gr), ("DRR", gr, gd)):
                out[name], st = c.count_triplets(x, y, **kw)
                tri += st["pairs"]  # in-range unordered triangles (XXY: per XX pair)
            out["_triangles"] = tri
            units = 0.0
        else:
            kw = dict(bins=req.bins, dmax=req.dmax, bpc=req.bpc, ani=req.kind == "2ani", stats=True)
            (dd, s1), (rr, s2), (dr, s3) = (c.count_pairs(gd, None, **kw), c.count_pairs(gr, None, **kw),
                                            c.count_pairs(gd, gr, **kw))
            out = {"DD": dd, "RR": rr, "DR": dr}
            units = s1["pairs"] + s2["pairs"] + s3["pairs"]
        out["_units"] = units
        return out


class PcfServer:
    def __init__(self, device: int = 0, slots: int = 4, hbm_budget: int | None = None,
                 cache_bytes: int = 8 << 30, max_wait_s: float = 0.05,
                 stuck_after_s: float | None = None, stuck_grace_s: float = 2.0,
                 watchdog_s: float = 0.01, slot_factory=None):
        """hbm_budget: bytes the running requests may hold at once (default:
        half the free device memory); cache_bytes: resident grids per slot;
        max_wait_s: a pending request older than this runs before shorter
        ones (bounds the wait that shortest-first scheduling adds);
        stuck_after_s: a request running longer than this has its slot
        aborted, and a slot that has not returned stuck_grace_s later is
        retired (None: no limit); watchdog_s: the watchdog's period;
        slot_factory(server, index): builds a slot (tests pass host-only
        stand-ins; default: a library context on `device`)."""
        self.max_wait_s = max_wait_s
        self.stuck_after_s = stuck_after_s
        self.stuck_grace_s = stuck_grace_s
        if hbm_budget is None:
            import torch
            free, _ = torch.cuda.mem_get_info(device)
            hbm_budget = int(free * 0.5)
        self.hbm_budget = hbm_budget
        self.catalogs: dict = {}
        self._lock = threading.Condition()
        self._pending: collections.deque = collections.deque()
        self._in_use = 0
        self._stop = False
        make = slot_factory or (lambda srv, i: _Slot(srv, i, device, cache_bytes))
        self.slots = [make(self, i) for i in range(slots)]
        self._threads = [threading.Thread(target=self._worker, args=(s,), daemon=True)
                         for s in self.slots]
        for t in self._threads:
            t.start()
        self._watchdog_s = watchdog_s
        self._watch = threading.Thread(target=self._watchdog, daemon=True)
        self._watch.start()

    # -- catalogs ----------------------------------------------------------
    def register(self, name: str, points: np.ndarray, box: float) -> None:
        """Keeps the catalog in page-locked host memory, so a slot's grid
        build copies it by DMA without staging it through the CPU."""
        import torch
        pts = api.as_points(points)
        pinned = torch.from_numpy(pts).pin_memory()
        self.catalogs[name] = {"points": pinned.numpy(), "box": float(box), "_pinned": pinned}

    # -- requests ----------------------------------------------------------
    def submit(self, req: Request) -> Future:
        req.t_submit = time.perf_counter()
        with self._lock:
            self._pending.append(req)
            self._lock.notify_all()
        return req.future

    def cancel(self, req: Request) -> bool:
        """Cancels a pending or running request; its future raises
        RequestCancelled.  Returns False if it had already completed."""
        with self._lock:
            if req.future.done():
                return False
            if req in self._pending:
                self._pending.remove(req)
                self._finish(req, exc=RequestCancelled(f"request {req.rid}"))
                return True
            req.stop_reason = RequestCancelled
            self._abort_slot_of(req)
            return True

    # -- failure handling (caller holds the lock) ---------------------------
    def _finish(self, req: Request, result=None, exc: BaseException | None = None) -> None:
        if req.future.done():
            return
        req.t_end = req.t_end or time.perf_counter()
        if exc is not None:
            req.future.set_exception(exc)
        else:
            req.future.set_result(result)

    def _abort_slot_of(self, req: Request) -> None:
        for sl in self.slots:
            if sl.current is req and not sl.aborted:
                sl.aborted = True
                try:
                    sl.abort(True)
                except Exception:  # pragma: no cover - the slot is failing anyway
                    pass

    def _watchdog(self) -> None:
        """Deadlines of pending and running requests, stuck slots."""
        while True:
            time.sleep(self._watchdog_s)
            with self._lock:
                if self._stop:
                    return
                now = time.perf_counter()
                for r in list(self._pending):
                    if r.deadline_s is not None and now > r.t_submit + r.deadline_s:
                        self._pending.remove(r)
                        self._finish(r, exc=DeadlineExceeded(f"request {r.rid} (pending)"))
                for sl in self.slots:
                    r = sl.current
                    if r is None or sl.retired:
                        continue
                    if r.deadline_s is not None and now > r.t_submit + r.deadline_s \
                            and r.stop_reason is None:
                        r.stop_reason = DeadlineExceeded
                        self._abort_slot_of(r)
                    if self.stuck_after_s is not None and now - r.t_start > self.stuck_after_s:
                        if r.stop_reason is None:
                            r.stop_reason = SlotStuck
                        self._abort_slot_of(r)
                        if now - r.t_start > self.stuck_after_s + self.stuck_grace_s:
                            # the slot did not come back from the abort: retire it
                            sl.retired = True
                            self._finish(r, exc=SlotStuck(f"slot {sl.idx}, request {r.rid}"))
                            self._lock.notify_all()

    def _admissible(self, req: Request) -> bool:
        """Admit while the running requests' footprints plus this one fit the
        budget (resident grid caches are bounded per slot by cache_bytes); a
        request that alone exceeds the budget runs when nothing else does."""
        sizes = {k: len(v["points"]) for k, v in self.catalogs.items()}
        need = request_bytes(req, sizes)
        return self._in_use + need <= self.hbm_budget or self._in_use == 0

    def _pick(self) -> Request | None:
        """Removes and returns the next request to run: among the admissible
        pending requests, one that has waited longer than max_wait_s (the
        oldest), else the one with the least expected work, so small
        requests do not queue behind large ones (shortest job first with an
        age bound).  Caller holds the lock."""
        now = time.perf_counter()
        best, best_i, best_cost = None, -1, None
        sizes = boxes = None
        for i, r in enumerate(self._pending):
            if not self._admissible(r):
                continue
            if now - r.t_submit > self.max_wait_s:
                best, best_i = r, i
                break
            if sizes is None:
                sizes = {k: len(v["points"]) for k, v in self.catalogs.items()}
                boxes = {k: v["box"] for k, v in self.catalogs.items()}
            cost = request_work(r, sizes, boxes)
            if best_cost is None or cost < best_cost:
                best, best_i, best_cost = r, i, cost
        if best is not None:
            del self._pending[best_i]
        return best

    def _worker(self, slot: _Slot) -> None:
        while True:
            with self._lock:
                req = None
                while req is None:
                    if self._stop or slot.retired:
                        return
                    req = self._pick()
                    if req is None:
                        self._lock.wait(0.05)
                sizes = {k: len(v["points"]) for k, v in self.catalogs.items()}
                fp = request_bytes(req, sizes)
                self._in_use += fp
                req.slot = slot.idx
                req.t_start = time.perf_counter()
                slot.current = req
            res, err = None, None
            try:
                res = slot.run(req)
            except Exception as e:  # reported to the caller, the slot keeps serving
                err = e
            with self._lock:
                req.t_end = time.perf_counter()
                slot.current = None
                if req.stop_reason is not None:
                    # stopped by cancel(), a deadline or the stuck-slot watchdog:
                    # whatever the call returned, the request failed for that reason
                    self._finish(req, exc=req.stop_reason(f"request {req.rid}"))
                elif err is not None:
                    self._finish(req, exc=err)
                else:
                    self._finish(req, result=res)
                if slot.aborted:
                    slot.aborted = False
                    try:
                        slot.abort(False)  # clear the request before the next call
                    except Exception:  # pragma: no cover
                        slot.retired = True
                self._in_use -= fp
                self._lock.notify_all()
                if slot.retired:
                    return

    def drop_grids(self) -> None:
        """Frees every slot's resident grids (their device memory returns to
        the slot's pool, so rebuilding them allocates nothing).  Call while
        no request runs."""
        for s in self.slots:
            for g, _ in s.cache.values():
                g.free()
            s.cache.clear()
            s.used = 0

    def close(self) -> None:
        with self._lock:
            self._stop = True
            self._lock.notify_all()
        for t in self._threads:
            t.join(timeout=5)
        self._watch.join(timeout=5)
        for s, t in zip(self.slots, self._threads):
            if t.is_alive():  # a retired slot still inside a call: leave its context
                continue
            for g, _ in getattr(s, "cache", {}).values():
                g.free()
            if hasattr(s, "ctx"):
                s.ctx.close()

    # -- a timed stream ----------------------------------------------------
    def run_stream(self, reqs: list[Request]) -> dict:
        """Submit requests at their arrival times; wait for all; report."""
        a0 = _lib.alloc_counters()
        t0 = time.perf_counter()
        for r in sorted(reqs, key=lambda r: r.arrival):
            delay = t0 + r.arrival - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            self.submit(r)
        results = [r.future.result() for r in reqs]
        t1 = time.perf_counter()
        return self._report(reqs, results, t1 - t0, a0)

    def run_serial(self, reqs: list[Request]) -> dict:
        """The plain per-call form of the same requests: one at a time, in
        arrival order, each submitted when the previous one has completed
        (no overlap on the device), and each gridding its catalogs from host
        memory (no resident grids kept between requests)."""
        a0 = _lib.alloc_counters()
        t0 = time.perf_counter()
        results = []
        for r in sorted(reqs, key=lambda r: r.arrival):
            results.append(self.submit(r).result())
            self.drop_grids()
        t1 = time.perf_counter()
        order = sorted(reqs, key=lambda r: r.arrival)
        return self._report(order, results, t1 - t0, a0)

    @staticmethod
    def _report(reqs, results, wall, allocs0=None) -> dict:
        lat = np.array([(r.t_end - r.t_submit) * 1e3 for r in reqs])
        units = sum(res.get("_units", 0.0) for res in results)
        tri = sum(res.get("_triangles", 0.0) for res in results)
        busy = {}
        for r in reqs:
            busy[r.kind] = busy.get(r.kind, 0.0) + (r.t_end - r.t_start)
        # how much the requests' device spans overlapped (continuous batching)
        spans = sorted((r.t_start, r.t_end) for r in reqs)
        overlap = sum(1 for (s0, e0), (s1, _) in zip(spans, spans[1:]) if s1 < e0)
        return {"requests": len(reqs), "wall_s": wall,
                "latency_ms": {"p50": float(np.percentile(lat, 50)),
                               "p99": float(np.percentile(lat, 99)),
                               "max": float(lat.max())},
                "pairs": units, "triangles": tri,
                "pairs_per_s": units / wall, "triplets_per_s": tri / wall,
                "overlapping_starts": overlap, "slot_seconds_by_kind": busy,
                "allocations": _alloc_delta(allocs0),
                "results": results}


def _alloc_delta(a0):
    """Library allocations (pcf_alloc_counters) since the counters `a0`."""
    if a0 is None:
        return None
    a1 = _lib.alloc_counters()
    return {k: a1[k] - a0[k] for k in a1}


def make_stream_mixed(n_requests: int, rate_hz: float, seed: int = 6000, n_max: int = 1_000_000,
                      n3_max: int = 65_536, box3: float = 1000.0, pool: int | None = None,
                      catalogs: bool = True) -> tuple[dict, list[Request]]:
    """The served-stream workload: Poisson arrivals of mixed requests, kinds
    2iso / 2ani / 3iso uniform, bins uniform in 20..50, dmax uniform in
    [40, 120], periodic or not by a seeded draw, over a seeded pool of
    catalog pairs (data clustered or uniform by a seeded draw, uniform
    randoms of the same size and box, unit weights) that the requests share,
    as requests of a survey share its catalogs: N log-uniform in [1e3, n_max],
    box 250 / 500 / 1000 (dmax < L/2 holds for all) for the 2-point pool;
    N in [1e3, n3_max], box3 (1000) for the 3iso pool, because a 3iso
    request costs N * (N dmax^3 / L^3)^2 and in the smaller boxes one
    65k-point request alone would take minutes.  pool: catalog pairs per
    pool (default n_requests / 4).  catalogs=False returns the same requests
    (other rate) without generating the catalogs again."""
    from . import catalog
    rng = np.random.default_rng(seed)
    npool = pool or max(4, n_requests // 4)
    cats = {}
    specs = {}
    for tag, cap in (("p", n_max), ("t", n3_max)):
        for j in range(npool):
            n = int(round(math.exp(rng.uniform(math.log(1e3), math.log(cap)))))
            box = box3 if tag == "t" else float(rng.choice([250.0, 500.0, 1000.0]))
            clustered = bool(rng.integers(0, 2))
            specs[(tag, j)] = (n, box, clustered)
    if catalogs:
        for (tag, j), (n, box, clustered) in specs.items():
            s0 = seed + 10 * j + (5 if tag == "t" else 0)
            gen = catalog.neyman_scott if clustered else catalog.uniform
            cats[f"{tag}d{j}"] = (gen(n, box, seed=s0), box)
            cats[f"{tag}r{j}"] = (catalog.uniform(n, box, seed=s0 + 1), box)
    reqs = []
    t = 0.0
    for i in range(n_requests):
        kind = KINDS[rng.integers(0, 3)]
        tag = "t" if kind == "3iso" else "p"
        j = int(rng.integers(0, npool))
        bins = int(rng.integers(20, 51))
        dmax = float(rng.uniform(40.0, 120.0))
        bpc = bool(rng.integers(0, 2))
        t += rng.exponential(1.0 / rate_hz)
        reqs.append(Request(kind, f"{tag}d{j}", f"{tag}r{j}", bins, dmax, bpc=bpc, arrival=t,
                            rid=i))
    return cats, reqs


def make_stream(n_requests: int, rate_hz: float, seed: int = 5000, n_max: int = 200_000,
                n3_max: int = 8_192) -> tuple[dict, list[Request]]:
    """A lighter seeded stream of mixed requests (kinds 2iso/2ani/3iso
    uniform, N log-uniform, bins 20-50 (3iso 10-20), dmax 40-120 with
    dmax < L/2 (3iso <= min(L/4, 60)), box 250/500/1000, clustered or
    uniform, unit weights, Poisson arrivals), N capped by n_max (n3_max for
    3iso): the request server's quick demonstration."""
    from . import catalog
    rng = np.random.default_rng(seed)
    cats, reqs = {}, []
    t = 0.0
    for i in range(n_requests):
        kind = KINDS[rng.integers(0, 3)]
        box = float(rng.choice([250.0, 500.0, 1000.0]))
        cap = n3_max if kind == "3iso" else n_max
        n = int(round(math.exp(rng.uniform(math.log(1e3), math.log(cap)))))
        bins = int(rng.integers(20, 51)) if kind != "3iso" else int(rng.integers(10, 21))
        dmax = float(rng.uniform(40.0, min(120.0, 0.45 * box)))
        if kind == "3iso":
            dmax = min(dmax, 0.25 * box, 60.0)
        clustered = bool(rng.integers(0, 2))
        dname, rname = f"d{i}", f"r{i}"
        gen = catalog.neyman_scott if clustered else catalog.uniform
        cats[dname] = (gen(n, box, seed=seed + 2 * i), box)
        cats[rname] = (catalog.uniform(n, box, seed=seed + 2 * i + 1), box)
        t += rng.exponential(1.0 / rate_hz)
        reqs.append(Request(kind, dname, rname, bins, dmax, bpc=bool(rng.integers(0, 2)),
                            arrival=t, rid=i))
    return cats, reqs


def main(argv=None):
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--requests", type=int, default=48)
    ap.add_argument("--rate", type=float, default=40.0)
    ap.add_argument("--slots", type=int, default=4)
    a = ap.parse_args(argv)
    cats, reqs = make_stream(a.requests, a.rate)
    srv = PcfServer(slots=a.slots)
    for k, (p, box) in cats.items():
        srv.register(k, p, box)
    try:
        rep = srv.run_stream(reqs)
    finally:
        srv.close()
    rep.pop("results")
    print(json.dumps(dict(rep, slots=a.slots, rate_hz=a.rate)))


if __name__ == "__main__":
    main()
