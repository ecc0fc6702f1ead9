"""GPU: the triplet kernel's flush budget and the queue control
(pcf_ctx_abort), with no device fault: nothing here traps, faults or waits
without a bound.  Aborted kernels stop taking work at their next work item
(they poll a word in mapped host memory) and the calls return
PCF_ERR_TIMEOUT; clearing the request makes the context usable again."""
import threading
import time

import numpy as np
import pytest

import oracle
from desi_b200 import api, catalog

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("budget", [1 << 12, 1])
@pytest.mark.parametrize("bpc", [False, True])
def test_triplet_flush_budget(budget, bpc):
    """A small budget flushes the per-CTA u32 histogram into the u64 global
    one many times per launch (1 << 12); budget 1 sends every anchor with more
    than one pair test to global atomics.  Both equal the oracle bit for bit
    (XXX and XXY)."""
    box, bins, dmax = 200.0, 12, 30.0
    D = catalog.neyman_scott(3000, box, seed=81, weights="unit")
    R = catalog.uniform(3200, box, seed=82, weights="unit")
    c = api.Context(0)
    try:
        c.set_option(api.PCF_OPT_TRIP_FLUSH_BUDGET, budget)
        gd, gr = c.grid(D, box), c.grid(R, box)
        for (x, y, X, Y) in ((gd, None, D, None), (gd, gr, D, R), (gr, gd, R, D)):
            got = c.count_triplets(x, y, bins=bins, dmax=dmax, bpc=bpc)
            want = oracle.triplets_iso(X, Y, box=box, bins=bins, dmax=dmax, bpc=bpc)
            assert want.sum() > 0
            assert np.array_equal(got, want)
    finally:
        c.close()


def _timeout(excinfo):
    return excinfo.value.status == api.PCF_ERR_TIMEOUT


def test_abort_refuses_calls_until_cleared(ctx):
    box = 250.0
    D = catalog.uniform(3000, box, seed=83)
    R = catalog.uniform(3100, box, seed=84)
    gd, gr = ctx.grid(D, box), ctx.grid(R, box)
    ctx.abort(True)
    try:
        with pytest.raises(api.PcfError) as e:
            ctx.count_pairs(gd, gr, bins=30, dmax=80.0)
        assert _timeout(e)
        with pytest.raises(api.PcfError) as e:
            ctx.count_triplets(gd, bins=10, dmax=30.0)
        assert _timeout(e)
        with pytest.raises(api.PcfError) as e:
            ctx.batch_pairs(gd, [gr], bins=30, dmax=80.0)
        assert _timeout(e)
    finally:
        ctx.abort(False)
    got = ctx.count_pairs(gd, gr, bins=30, dmax=80.0)
    assert np.array_equal(got, oracle.pairs(D, R, box=box, bins=30, dmax=80.0))


def test_kernels_poll_the_abort_word():
    """With the host's own check off, the launches run and the persistent
    kernels themselves see the request at their next ticket or anchor: the
    calls report PCF_ERR_TIMEOUT (device-output calls through synchronize)."""
    import torch
    box = 250.0
    D = catalog.neyman_scott(20000, box, seed=85, weights="uniform")
    R = catalog.uniform(20000, box, seed=86, weights="uniform")
    c = api.Context(0)
    try:
        gd, gr = c.grid(D, box), c.grid(R, box)
        c.set_option(api.PCF_OPT_ABORT_HOST_CHECK, 0)
        c.abort(True)
        for call in (lambda: c.count_pairs(gd, gr, bins=30, dmax=80.0, bpc=True),
                     lambda: c.count_pairs(gd, None, bins=30, dmax=80.0, ani=True, stats=True),
                     lambda: c.count_triplets(gd, gr, bins=10, dmax=30.0),
                     lambda: c.batch_pairs(gd, [gr], bins=30, dmax=80.0)):
            with pytest.raises(api.PcfError) as e:
                call()
            assert _timeout(e)
        out = torch.zeros(30, dtype=torch.float64, device="cuda")
        c.count_pairs(gd, gr, bins=30, dmax=80.0, out_device_ptr=out.data_ptr())
        with pytest.raises(api.PcfError) as e:
            c.synchronize()
        assert _timeout(e)
        c.abort(False)
        c.set_option(api.PCF_OPT_ABORT_HOST_CHECK, 1)
        got = c.count_pairs(gd, gr, bins=30, dmax=80.0, bpc=True)
        want = oracle.pairs(D, R, box=box, bins=30, dmax=80.0, bpc=True)
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=0)
        c.synchronize()
    finally:
        c.close()


def test_abort_from_another_thread_stops_a_running_call():
    """A long triplet launch (periodic 3iso, 65536 clustered points) is
    stopped by pcf_ctx_abort from a second host thread: the call returns
    PCF_ERR_TIMEOUT in a fraction of its full duration, and the context
    then counts a small case exactly."""
    box = 250.0
    D = catalog.neyman_scott(65536, box, seed=87, weights="unit")
    c = api.Context(0)
    try:
        g = c.grid(D, box)
        t0 = time.perf_counter()
        c.count_triplets(g, bins=30, dmax=80.0, bpc=True)
        full = time.perf_counter() - t0
        timer = threading.Timer(full / 5, lambda: c.abort(True))
        t0 = time.perf_counter()
        timer.start()
        with pytest.raises(api.PcfError) as e:
            c.count_triplets(g, bins=30, dmax=80.0, bpc=True)
        took = time.perf_counter() - t0
        timer.join()
        assert _timeout(e)
        assert took < 0.6 * full, (took, full)
        c.abort(False)
        small = catalog.uniform(2000, box, seed=88)
        gs = c.grid(small, box)
        assert np.array_equal(c.count_triplets(gs, bins=10, dmax=30.0),
                              oracle.triplets_iso(small, box=box, bins=10, dmax=30.0))
    finally:
        c.abort(False)
        c.close()
