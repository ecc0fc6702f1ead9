"""GPU: the 3-point histograms of one data catalog against random catalogs
of uneven sizes in one persistent launch (pcf_batch_triplets) equal the
per-call histograms and the FP64 oracle: bit for bit with unit weights,
within 1e-12 relative with weights."""
import numpy as np
import pytest

import oracle
from desi_b200 import api, catalog

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("bpc", [False, True])
@pytest.mark.parametrize("w", ["unit", "uniform"])
def test_batch_triplets_equal_per_call_and_oracle(ctx, bpc, w):
    box, bins, dmax = 200.0, 12, 30.0
    D = catalog.neyman_scott(2500, box, seed=91, weights=w)
    Rs = [catalog.uniform(n, box, seed=92 + i, weights=w) for i, n in enumerate((900, 3100, 1700))]
    gd = ctx.grid(D, box)
    grs = [ctx.grid(R, box) for R in Rs]
    (ddd, rrr, ddr, drr), st = ctx.batch_triplets(gd, grs, bins=bins, dmax=dmax, bpc=bpc, stats=True)
    assert st["pairs"] > 0
    if w == "unit":
        cmp = np.testing.assert_array_equal
    else:
        cmp = lambda a, b: np.testing.assert_allclose(a, b, rtol=1e-12, atol=0)  # noqa: E731
    kw = dict(bins=bins, dmax=dmax, bpc=bpc)
    okw = dict(box=box, bins=bins, dmax=dmax, bpc=bpc)
    cmp(ddd, ctx.count_triplets(gd, **kw))
    cmp(ddd, oracle.triplets_iso(D, **okw))
    for i, (g, R) in enumerate(zip(grs, Rs)):
        cmp(rrr[i], ctx.count_triplets(g, **kw))
        cmp(ddr[i], ctx.count_triplets(gd, g, **kw))
        cmp(drr[i], ctx.count_triplets(g, gd, **kw))
        cmp(rrr[i], oracle.triplets_iso(R, **okw))
        cmp(ddr[i], oracle.triplets_iso(D, R, **okw))
        cmp(drr[i], oracle.triplets_iso(R, D, **okw))


def test_batch_triplets_flush_budget_and_abort():
    """The batch flushes a CTA's shared histogram when it crosses into the
    next job and before the flush budget; an abort request stops it."""
    box, bins, dmax = 200.0, 10, 28.0
    D = catalog.neyman_scott(2200, box, seed=95)
    Rs = [catalog.uniform(n, box, seed=96 + i) for i, n in enumerate((1500, 2600))]
    c = api.Context(0)
    try:
        c.set_option(api.PCF_OPT_TRIP_FLUSH_BUDGET, 1 << 11)
        gd = c.grid(D, box)
        grs = [c.grid(R, box) for R in Rs]
        ddd, rrr, ddr, drr = c.batch_triplets(gd, grs, bins=bins, dmax=dmax, bpc=True)
        okw = dict(box=box, bins=bins, dmax=dmax, bpc=True)
        assert np.array_equal(ddd, oracle.triplets_iso(D, **okw))
        for i, R in enumerate(Rs):
            assert np.array_equal(rrr[i], oracle.triplets_iso(R, **okw))
            assert np.array_equal(ddr[i], oracle.triplets_iso(D, R, **okw))
            assert np.array_equal(drr[i], oracle.triplets_iso(R, D, **okw))
        c.set_option(api.PCF_OPT_ABORT_HOST_CHECK, 0)
        c.abort(True)
        with pytest.raises(api.PcfError) as e:
            c.batch_triplets(gd, grs, bins=bins, dmax=dmax, bpc=True)
        assert e.value.status == api.PCF_ERR_TIMEOUT
        c.abort(False)
        again = c.batch_triplets(gd, grs, bins=bins, dmax=dmax, bpc=True)
        assert np.array_equal(again[0], ddd)
    finally:
        c.close()
