"""GPU: the continuous-batching server gives every request the same
histograms alone and in the mix (unit weights: bit-exact), admits by HBM
footprint, and reuses resident grids."""
import numpy as np
import pytest

from desi_b200 import catalog

pytestmark = pytest.mark.gpu


def _requests():
    from desi_b200.serve import Request
    reqs = []
    spec = [("2iso", 30, 40.0, False), ("2ani", 20, 35.0, True), ("3iso", 10, 20.0, False),
            ("2iso", 25, 60.0, True), ("3iso", 8, 25.0, True), ("2ani", 30, 50.0, False),
            ("2iso", 40, 45.0, False), ("3iso", 12, 18.0, False)]
    for i, (k, b, d, bpc) in enumerate(spec):
        reqs.append(Request(k, f"d{i % 3}", f"r{i % 2}", b, d, bpc=bpc, arrival=0.002 * i, rid=i))
    return reqs


def _server(slots, budget=None):
    from desi_b200.serve import PcfServer
    srv = PcfServer(slots=slots, hbm_budget=budget)
    for i in range(3):
        srv.register(f"d{i}", catalog.neyman_scott(3000 + 700 * i, 200.0, seed=90 + i), 200.0)
    for i in range(2):
        srv.register(f"r{i}", catalog.uniform(3500 + 500 * i, 200.0, seed=95 + i), 200.0)
    return srv


def test_same_result_alone_and_in_the_mix():
    alone = _server(1)
    try:
        solo = []
        for r in _requests():  # one at a time
            solo.append(alone.submit(r).result())
    finally:
        alone.close()
    mix = _server(4)
    try:
        rep = mix.run_stream(_requests())
    finally:
        mix.close()
    assert rep["requests"] == len(solo)
    for a, b in zip(solo, rep["results"]):
        assert a.keys() == b.keys()
        for k in a:
            assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k
    # the mix really ran requests at the same time on the device
    assert rep["overlapping_starts"] > 0


def test_mix_equals_the_oracle():
    """The histograms of requests served in the mix equal the FP64 oracle
    (unit weights: bit for bit), for the 2-point and 3-point kinds."""
    import oracle
    reqs = _requests()
    mix = _server(4)
    try:
        cats = {k: v["points"] for k, v in mix.catalogs.items()}
        rep = mix.run_stream(reqs)
    finally:
        mix.close()
    for r, res in zip(reqs, rep["results"]):
        D, R = cats[r.data], cats[r.rand]
        kw = dict(box=200.0, bins=r.bins, dmax=r.dmax, bpc=r.bpc)
        if r.kind == "3iso":
            assert np.array_equal(res["DDD"], oracle.triplets_iso(D, **kw))
            assert np.array_equal(res["DDR"], oracle.triplets_iso(D, R, **kw))
        else:
            ani = r.kind == "2ani"
            assert np.array_equal(res["DD"], oracle.pairs(D, ani=ani, **kw))
            assert np.array_equal(res["DR"], oracle.pairs(D, R, ani=ani, **kw))


def test_admission_by_footprint_serialises_but_completes():
    srv = _server(4, budget=1)  # no two requests fit together
    try:
        reqs = _requests()[:4]
        rep = srv.run_stream(reqs)
        assert rep["requests"] == 4
        spans = sorted((r.t_start, r.t_end) for r in reqs)
        for (s0, e0), (s1, e1) in zip(spans, spans[1:]):
            assert s1 >= e0  # never two at once
    finally:
        srv.close()


def test_dropped_grids_rebuild_to_the_same_result():
    """drop_grids frees the resident grids; the next pass grids the catalogs
    again (from the slots' pools) and returns identical histograms."""
    srv = _server(2)
    try:
        first = srv.run_stream(_requests()[:5])["results"]
        assert any(s.cache for s in srv.slots)
        srv.drop_grids()
        assert all(not s.cache and s.used == 0 for s in srv.slots)
        again = srv.run_stream(_requests()[:5])["results"]
    finally:
        srv.close()
    for a, b in zip(first, again):
        for k in a:
            assert np.array_equal(np.asarray(a[k]), np.asarray(b[k])), k

