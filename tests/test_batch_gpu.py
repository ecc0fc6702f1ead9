"""GPU: one data catalog against random catalogs of uneven sizes in one
persistent launch (pcf_batch_pairs, the -rd mode), plain and graph-replayed,
equals the per-call histograms (bit-exact unit weights, rtol 1e-12 weighted)."""
import numpy as np
import pytest

from desi_b200 import catalog

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("ani", [False, True, "both"])
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
        cmp1 = (lambda a, b: np.testing.assert_allclose(a, b, rtol=1e-12, atol=0)) if w != "unit" \
            else (lambda a, b: np.testing.assert_array_equal(a, b))
        cmp = (lambda a, b: [cmp1(x, y) for x, y in zip(a, b)]) if ani == "both" else cmp1
        at = (lambda h, i: (h[0][i], h[1][i])) if ani == "both" else (lambda h, i: h[i])
        cmp(dd, ctx.count_pairs(gd, None, bins=bins, dmax=dmax, ani=ani, bpc=bpc))
        for i, g in enumerate(grs):
            cmp(at(rr, i), ctx.count_pairs(g, None, bins=bins, dmax=dmax, ani=ani, bpc=bpc))
            cmp(at(dr, i), ctx.count_pairs(gd, g, bins=bins, dmax=dmax, ani=ani, bpc=bpc))


@pytest.mark.parametrize("w", ["uniform", "signed"])
def test_batch_both_kinds(ctx, w):
    """ani="both" in a batch equals the single-kind per-call histograms, for
    exact (fixed-point) and signed (FP64) weights.  The batch runs as two
    single-kind batches (work_items: one per job slot of each)."""
    box, bins, dmax = 300.0, 16, 40.0
    rng = np.random.default_rng(80)
    def wts(P):
        if w == "signed":
            P = P.copy()
            P[:, 3] = rng.uniform(-1.0, 1.0, len(P)).astype(np.float32)
        return P
    D = wts(catalog.neyman_scott(3000, box, seed=81, weights="uniform"))
    Rs = [wts(catalog.uniform(n, box, seed=82 + i, weights="uniform")) for i, n in enumerate([2500, 400, 5000])]
    gd = ctx.grid(D, box)
    grs = [ctx.grid(R, box) for R in Rs]
    (dd, rr, dr), st = ctx.batch_pairs(gd, grs, bins=bins, dmax=dmax, ani="both", bpc=True, stats=True)
    slots = 1 + 2 * len(grs)
    assert st["work_items"] == 2 * slots
    def cmp(a, b):
        assert np.all(np.abs(a - b) <= 1e-12 * (np.abs(b) + (1.0 if w == "signed" else 0.0)))
    for k, is_ani in enumerate((False, True)):
        cmp(dd[k], ctx.count_pairs(gd, None, bins=bins, dmax=dmax, ani=is_ani, bpc=True))
        for i, g in enumerate(grs):
            cmp(rr[k][i], ctx.count_pairs(g, None, bins=bins, dmax=dmax, ani=is_ani, bpc=True))
            cmp(dr[k][i], ctx.count_pairs(gd, g, bins=bins, dmax=dmax, ani=is_ani, bpc=True))


def test_autotune_and_estimator(ctx, tmp_path):
    import oracle
    box, bins, dmax = 250.0, 30, 80.0
    D = catalog.neyman_scott(6000, box, seed=111)
    R = catalog.uniform(6000, box, seed=112)
    gd, gr = ctx.grid(D, box), ctx.grid(R, box)
    res = ctx.autotune_pairs(gd, gr, bins=bins, dmax=dmax, bpc=True)
    assert res["tried"] >= 12 and res["best_ms"] <= res["default_ms"] + 1e-6
    assert res["tile"] in (16, 32) and res["chunk"] in (1, 4, 8)
    assert ctx.tune_size == 1
    # counts with the tuned shape still match the oracle bit for bit
    dr = ctx.count_pairs(gd, gr, bins=bins, dmax=dmax, bpc=True)
    assert np.array_equal(dr, oracle.pairs(D, R, box=box, bins=bins, dmax=dmax, bpc=True))
    p = str(tmp_path / "tune.txt")
    ctx.tune_save(p)
    assert len(open(p).read().split()) == 6  # key refine hist_mode ms tile chunk
    from desi_b200 import api
    c2 = api.Context(0)
    c2.tune_load(p)
    assert c2.tune_size == 1
    # Landy-Szalay as the reference's script computes it
    dd = ctx.count_pairs(gd, None, bins=bins, dmax=dmax, bpc=True)
    rr = ctx.count_pairs(gr, None, bins=bins, dmax=dmax, bpc=True)
    xi = c2.estimate((dd, dr, rr))
    DD, DR, RR = (np.where(h == 0, 1e-11, h) for h in (dd, dr, rr))
    np.testing.assert_allclose(xi, (DD - 2 * DR + RR) / RR, rtol=1e-14)
    z = c2.estimate((dd, dr, rr), n_d=6000, n_r=6000)
    n = 6000.0
    want = (DD / (n * (n - 1)) - 2 * DR / (n * n) + RR / (n * (n - 1))) / (RR / (n * (n - 1)))
    np.testing.assert_allclose(z, want, rtol=1e-12)
    c2.close()
