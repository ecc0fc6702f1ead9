"""GPU parity of the analytic periodic-box histograms (RR of 2iso -bpc -a;
DDR/RRR of 3iso -bpc -a) against the FP64 oracle, rtol 1e-10."""
import numpy as np
import pytest

import oracle
from desi_b200 import catalog

pytestmark = pytest.mark.gpu
RTOL = 1e-10


@pytest.mark.parametrize("bins,n,box,dmax", [(30, 32768, 250.0, 80.0), (20, 5000, 100.0, 33.3),
                                              (40000, 1000, 1000.0, 400.0)])
@pytest.mark.parametrize("wrap", [True, False])
def test_analytic_rr(ctx, bins, n, box, dmax, wrap):
    got = ctx.analytic_rr(bins, n, box, dmax, wrap=wrap)
    want = oracle.analytic_rr(bins, n, box, dmax, wrap=wrap)
    np.testing.assert_allclose(got, want, rtol=1e-15, atol=0)


@pytest.mark.parametrize("clu", [False, True])
def test_analytic_3iso_small_subgrid(ctx, clu):
    box, bins, dmax, ptt, bn_ref = 100.0, 8, 30.0, 10, 8
    gen = catalog.neyman_scott if clu else catalog.uniform
    D = gen(1500, box, seed=51)
    g = ctx.grid(D, box)
    ddd, ddr, rrr = ctx.analytic_3iso(g, bins=bins, dmax=dmax, ptt=ptt, bn_ref=bn_ref)
    oddr, orrr, _, _ = oracle.analytic_3iso(D, box=box, bins=bins, dmax=dmax, ptt=ptt,
                                            bn_ref=bn_ref)
    np.testing.assert_allclose(rrr, orrr, rtol=RTOL, atol=1e-12 * np.abs(orrr).max())
    np.testing.assert_allclose(ddr, oddr, rtol=RTOL, atol=1e-12 * np.abs(oddr).max())
    assert np.array_equal(ddd, oracle.triplets_iso(D, box=box, bins=bins, dmax=dmax, bpc=True))


def test_analytic_3iso_reference_subgrid_selected_bins(ctx):
    """The reference's own sub-binning (ptt 100, bn_ref 200) on partial bins."""
    box, bins, dmax = 100.0, 6, 30.0
    D = catalog.uniform(2000, box, seed=52)
    g = ctx.grid(D, box)
    _, ddr, rrr = ctx.analytic_3iso(g, bins=bins, dmax=dmax, ptt=100, bn_ref=200, with_ddd=False)
    ff, ffr, alpha_ref = oracle.analytic_ff(D, box=box, bins=bins, dmax=dmax, ptt=100, bn_ref=200)
    checked = 0
    for (i, j, k) in [(0, 0, 1), (1, 2, 4), (2, 2, 5), (0, 3, 3), (5, 0, 5), (3, 1, 2)]:
        v, r, d = oracle.analytic_bin(i, j, k, bins=bins, dmax=dmax, bn_ref=200,
                                      alpha_ref=alpha_ref, ff_ref=ffr)
        if 0 < v < 8:
            np.testing.assert_allclose(rrr[i, j, k], r, rtol=RTOL)
            np.testing.assert_allclose(ddr[i, j, k], d, rtol=RTOL)
            checked += 1
    assert checked >= 3
