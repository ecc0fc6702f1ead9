"""CPU: the served leg of bench.py (run_served) with a stand-in server: one
warm-up pass, then served and plain passes interleaved three times, the best
of each form kept, then the Poisson pass at 70% of the best served capacity;
the reported ratio is best served pairs/s over best plain pairs/s."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


class _Req:
    def __init__(self):
        self.arrival = 0.0


def test_served_leg_interleaves_and_keeps_the_best(monkeypatch):
    import bench
    from desi_b200 import serve

    calls = []
    walls = {"stream": iter([9.0, 3.0, 2.0, 2.5, 4.0]), "serial": iter([3.5, 2.2, 2.4])}

    def rep(kind):
        w = next(walls[kind])
        return {"wall_s": w, "pairs_per_s": 100.0 / w, "triplets_per_s": 10.0 / w,
                "overlapping_starts": 1, "latency_ms": {"p50": 1.0, "p99": 2.0, "max": 3.0},
                "allocations": {"device_allocs": 0}, "results": []}

    class FakeServer:
        def __init__(self, slots):
            assert slots == 4

        def register(self, name, points, box):
            pass

        def drop_grids(self):
            calls.append("drop")

        def run_stream(self, reqs):
            calls.append("stream")
            return rep("stream")

        def run_serial(self, reqs):
            calls.append("serial")
            return rep("serial")

        def close(self):
            calls.append("close")

    monkeypatch.setattr(serve, "PcfServer", FakeServer)
    monkeypatch.setattr(serve, "make_stream_mixed",
                        lambda n, rate_hz, catalogs=True: ({}, [_Req() for _ in range(n)]))
    out = bench.run_served(n_requests=10)
    passes = [c for c in calls if c in ("stream", "serial")]
    assert passes == ["stream"] + ["stream", "serial"] * 3 + ["stream"]
    assert calls[-1] == "close"
    assert out["closed_loop"]["passes_wall_s"] == [3.0, 2.0, 2.5]
    assert out["plain_passes_wall_s"] == [3.5, 2.2, 2.4]
    assert abs(out["served_vs_plain"]["pairs_per_s"] - (100 / 2.0) / (100 / 2.2)) < 1e-12
    assert abs(out["capacity_req_per_s"] - 10 / 2.0) < 1e-12
    assert abs(out["rate_hz"] - 0.7 * 10 / 2.0) < 1e-12


def test_served_leg_runs_in_a_fresh_process_or_falls_back(monkeypatch):
    """run_served_isolated reads the child's JSON report; when the child
    fails it runs the leg in the bench process and says why."""
    import subprocess

    import bench

    class Done:
        returncode = 0
        stdout = 'noise\n{"served_vs_plain": {"pairs_per_s": 1.09}}\n'
        stderr = ""

    seen = []

    def ok_run(cmd, capture_output, text, timeout, cwd):
        seen.append(cmd)
        return Done()

    monkeypatch.setattr(subprocess, "run", ok_run)
    rep = bench.run_served_isolated(12)
    assert rep["served_vs_plain"]["pairs_per_s"] == 1.09
    assert rep["process"].startswith("fresh process")
    assert seen[0][0] == sys.executable and "run_served(12)" in seen[0][2]

    class Failed(Done):
        returncode = 1
        stdout = ""
        stderr = "no device"

    monkeypatch.setattr(subprocess, "run", lambda *a, **k: Failed())
    monkeypatch.setattr(bench, "run_served", lambda n: {"served_vs_plain": {"pairs_per_s": 0.9}})
    rep = bench.run_served_isolated(12)
    assert rep["served_vs_plain"]["pairs_per_s"] == 0.9
    assert "child exited 1" in rep["process"] and "no device" in rep["process"]
