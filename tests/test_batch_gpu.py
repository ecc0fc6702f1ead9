"""GPU: one data catalog against random catalogs of uneven sizes in one
persistent launch (pcf_batch_pairs, the -rd mode), plain and graph-replayed,
equals the per-call histograms (bit-exact unit weights, rtol 1e-12 weighted)."""
import numpy as np
import pytest

from desi_b200 import catalog

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ani", [False, True])
@pytest.mark.parametrize("bpc", [False, True])
@pytest.mark.parametrize("w", ["unit", "uniform"])
@pytest.mark.parametrize("graph", [False, True])
def test_batch_equals_per_call(ctx, ani, bpc, w, graph):
    box, bins, dmax = 300.0, 16, 40.0
    D = catalog.neyman_scott(4000, box, seed=71, weights=w)
    sizes = [500, 3000, 1200, 7000, 90]
    Rs = [catalog.uniform(n, box, seed=72 + i, weights=w) for i, n in enumerate(sizes)]
    gd = ctx.grid(D, box)
    grs = [ctx.grid(R, box) for R in Rs]
    reps = 3 if graph else 1
    for _ in range(reps):  # graph: captured on the first call, replayed after
        (dd, rr, dr), st = ctx.batch_pairs(gd, grs, bins=bins, dmax=dmax, ani=ani, bpc=bpc,
                                           graph=graph, stats=True)
        cmp = (lambda a, b: np.testing.assert_allclose(a, b, rtol=1e-12, atol=0)) if w != "unit" \
            else (lambda a, b: np.testing.assert_array_equal(a, b))
        cmp(dd, ctx.count_pairs(gd, None, bins=bins, dmax=dmax, ani=ani, bpc=bpc))
        for i, g in enumerate(grs):
            cmp(rr[i], ctx.count_pairs(g, None, bins=bins, dmax=dmax, ani=ani, bpc=bpc))
            cmp(dr[i], ctx.count_pairs(gd, g, bins=bins, dmax=dmax, ani=ani, bpc=bpc))
