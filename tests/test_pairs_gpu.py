"""GPU parity of the pair histograms against the FP64 oracle.

Unit weights: bit-exact.  Weighted: |gpu - oracle| <= 1e-12 * |oracle|
(FP64 sums in a different order).
"""
import numpy as np
import pytest

import oracle
from desi_b200 import catalog

pytestmark = pytest.mark.gpu
RTOL_W = 1e-12


def _cmp(got, want, weighted):
    if weighted:
        np.testing.assert_allclose(got, want, rtol=RTOL_W, atol=0)
    else:
        assert np.array_equal(got, want), (np.abs(got - want).max(), np.argwhere(got != want)[:5])


CASES = [
    # (name, n, box, bins, dmax, clustered, weights)
    ("uniform", 3000, 250.0, 30, 80.0, False, "unit"),
    ("clustered", 3000, 250.0, 30, 80.0, True, "unit"),
    ("weighted", 2500, 250.0, 30, 80.0, True, "uniform"),
    ("odd", 2000, 173.0, 17, 41.3, False, "unit"),
]


@pytest.mark.parametrize("name,n,box,bins,dmax,clu,w", CASES)
@pytest.mark.parametrize("ani", [False, True])
@pytest.mark.parametrize("bpc", [False, True])
def test_pairs_xx_xy(ctx, name, n, box, bins, dmax, clu, w, ani, bpc):
    gen = catalog.neyman_scott if clu else catalog.uniform
    D = gen(n, box, seed=11, weights=w)
    R = catalog.uniform(n + 123, box, seed=12, weights=w)
    gd, gr = ctx.grid(D, box), ctx.grid(R, box)
    weighted = w != "unit"
    for (a, b, A, B) in ((gd, None, D, None), (gr, None, R, None), (gd, gr, D, R)):
        got = ctx.count_pairs(a, b, bins=bins, dmax=dmax, ani=ani, bpc=bpc)
        want = oracle.pairs(A, B, box=box, bins=bins, dmax=dmax, ani=ani, bpc=bpc)
        _cmp(got, want, weighted)


def test_reference_catalogs_1k(ctx, catalogs):
    D, R = catalogs["data_1K"], catalogs["rand0_1K"]
    box = 251.0
    gd, gr = ctx.grid(D, box), ctx.grid(R, box)
    for ani in (False, True):
        for bpc in (False, True):
            for a, b, A, B in ((gd, None, D, None), (gd, gr, D, R)):
                got = ctx.count_pairs(a, b, bins=30, dmax=80.0, ani=ani, bpc=bpc)
                want = oracle.pairs(A, B, box=box, bins=30, dmax=80.0, ani=ani, bpc=bpc)
                _cmp(got, want, False)


def test_lattice_exact_edges(ctx):
    """Integer lattice: many separations sit exactly on bin edges and on dmax."""
    g = np.stack(np.meshgrid(np.arange(12), np.arange(12), np.arange(12), indexing="ij"), -1)
    pts = np.concatenate([g.reshape(-1, 3).astype(np.float32) * 2.5 + 0.25,
                          np.ones((12 ** 3, 1), np.float32)], 1)
    box = 30.0
    gd = ctx.grid(pts, box)
    for ani in (False, True):
        for bpc, dmax in ((False, 10.0), (True, 10.0), (False, 12.5)):
            for bins in (10, 20, 4):
                got = ctx.count_pairs(gd, None, bins=bins, dmax=dmax, ani=ani, bpc=bpc)
                want = oracle.pairs(pts, None, box=box, bins=bins, dmax=dmax, ani=ani, bpc=bpc)
                _cmp(got, want, False)


def test_duplicates_and_zero_separation(ctx):
    rng = np.random.default_rng(3)
    base = catalog.uniform(400, 100.0, seed=4)
    pts = np.concatenate([base, base[:50], base[:10]])  # exact duplicates
    pts = pts[rng.permutation(len(pts))]
    other = np.concatenate([base[100:160], catalog.uniform(200, 100.0, seed=5)])
    box = 100.0
    a, b = ctx.grid(pts, box), ctx.grid(other, box)
    for ani in (False, True):
        for bpc in (False, True):
            got = ctx.count_pairs(a, None, bins=25, dmax=30.0, ani=ani, bpc=bpc)
            want = oracle.pairs(pts, None, box=box, bins=25, dmax=30.0, ani=ani, bpc=bpc)
            _cmp(got, want, False)
            got = ctx.count_pairs(a, b, bins=25, dmax=30.0, ani=ani, bpc=bpc)
            want = oracle.pairs(pts, other, box=box, bins=25, dmax=30.0, ani=ani, bpc=bpc)
            _cmp(got, want, False)


def test_ds_exact_and_wide_bins(ctx):
    D = catalog.uniform(1500, 200.0, seed=7)
    g = ctx.grid(D, 200.0)
    from desi_b200.api import PCF_DS_EXACT
    got = ctx.count_pairs(g, None, bins=40, dmax=60.0, bpc=True, flags=PCF_DS_EXACT)
    want = oracle.pairs(D, None, box=200.0, bins=40, dmax=60.0, bpc=True, ds_exact=True)
    _cmp(got, want, False)
    got = ctx.count_pairs(g, None, bins=700, dmax=60.0)
    want = oracle.pairs(D, None, box=200.0, bins=700, dmax=60.0)
    _cmp(got, want, False)


def test_tiny_catalogs(ctx):
    one = np.array([[1.0, 2.0, 3.0, 1.0]], np.float32)
    two = np.array([[1.0, 2.0, 3.0, 1.0], [4.0, 2.0, 3.0, 1.0]], np.float32)
    g1, g2 = ctx.grid(one, 10.0), ctx.grid(two, 10.0)
    assert ctx.count_pairs(g1, None, bins=5, dmax=4.0).sum() == 0
    h = ctx.count_pairs(g2, None, bins=5, dmax=4.0)
    assert h[3] == 2 and h.sum() == 2
    h = ctx.count_pairs(g1, g2, bins=5, dmax=4.0)
    assert h[0] == 1 and h[3] == 1


def test_out_of_box_rejected(ctx):
    from desi_b200.api import PcfError
    bad = np.array([[1.0, 2.0, 10.0, 1.0]], np.float32)
    with pytest.raises(PcfError):
        ctx.grid(bad, 10.0)


def test_bpc_dmax_limit(ctx):
    from desi_b200.api import PcfError
    g = ctx.grid(catalog.uniform(100, 10.0, seed=1), 10.0)
    with pytest.raises(PcfError):
        ctx.count_pairs(g, None, bins=5, dmax=5.0, bpc=True)


def test_grid_is_a_permutation_in_cell_order(ctx):
    D = catalog.neyman_scott(5000, 250.0, seed=9)
    g = ctx.grid(D, 250.0, partitions=17)
    pts, cs = g.download()
    assert cs[0] == 0 and cs[-1] == len(D) and np.all(np.diff(cs) >= 0)
    key = lambda a: np.lexsort(a[:, :3].T)
    assert np.array_equal(pts[key(pts)], D[key(D)])
    P = 17
    cell = np.float32(250.0) / np.float32(P)
    idx = np.minimum((pts[:, :3] / cell).astype(np.int64), P - 1)
    cid = (idx[:, 0] * P + idx[:, 1]) * P + idx[:, 2]
    assert np.all(np.diff(cid) >= 0)


def _cell_table(D, box, P):
    cell = np.float32(box) / np.float32(P)
    idx = np.clip((D[:, :3] / cell).astype(np.int64), 0, P - 1)
    cid = (idx[:, 0] * P + idx[:, 1]) * P + idx[:, 2]
    return np.concatenate([[0], np.cumsum(np.bincount(cid, minlength=P ** 3))]), cid


@pytest.mark.parametrize("build", [1, 2])
@pytest.mark.parametrize("case", ["odd_small", "one_cell", "dense_cell", "large", "per_point"])
def test_grid_build_cases(ctx, case, build):
    """Both grid builds (PCF_OPT_GRID_BUILD 1: per-point, 2: bucketed; the
    default picks by size) against a host counting sort: the cell table, the
    multiset of points in cell order, and (through the pair-packed blocks
    and integer weights) DD against the oracle.  odd_small: an odd catalog
    in many small buckets (pair blocks straddle buckets and cluster shares);
    one_cell: every point in a single bucket larger than a cluster sorts in
    shared memory; dense_cell: 20000 points inside one cell beside a uniform
    background; large: 2M points in 64^3 cells; per_point: 300^3 cells, more
    buckets than the bucketed build's shared arrays hold, so the per-point
    build runs either way."""
    from desi_b200.api import PCF_OPT_GRID_BUILD
    ctx.set_option(PCF_OPT_GRID_BUILD, build)
    try:
        _grid_build_case(ctx, case)
    finally:
        ctx.set_option(PCF_OPT_GRID_BUILD, 0)


def _grid_build_case(ctx, case):
    rng = np.random.default_rng(5)
    box = 100.0
    if case == "odd_small":
        D, P = catalog.uniform(3001, box, seed=3, weights="uniform"), 9
    elif case == "one_cell":
        D, P = catalog.uniform(14001, box, seed=7, weights="uniform"), 1
    elif case == "dense_cell":
        bg = catalog.uniform(5001, box, seed=4, weights="uniform")
        dense = bg[:1].repeat(20000, 0)
        dense[:, :3] = rng.uniform(40.5, 49.5, size=(20000, 3)).astype(np.float32)
        D, P = np.ascontiguousarray(np.concatenate([bg, dense])), 10
    elif case == "large":
        D, P = catalog.uniform(1 << 21, box, seed=6), 64
    else:
        D, P = catalog.uniform(200001, box, seed=8, weights="uniform"), 300
    g = ctx.grid(D, box, partitions=P)
    pts, cs = g.download()
    want_cs, cid = _cell_table(D, box, P)
    assert np.array_equal(cs, want_cs)
    key = lambda a: np.lexsort(a.T)
    assert np.array_equal(pts[key(pts)], D[key(D)])
    _, cid_out = _cell_table(pts, box, P)
    assert np.all(np.diff(cid_out) >= 0)
    if case == "per_point":  # counts on the 300^3 cells themselves (the grid's partitions)
        got = ctx.count_pairs(g, None, bins=5, dmax=1.0)
        want = oracle.pairs(D, None, box=box, bins=5, dmax=1.0)
        np.testing.assert_allclose(got, want, rtol=RTOL_W, atol=0)
    elif case != "large":
        got = ctx.count_pairs(g, None, bins=12, dmax=30.0)
        want = oracle.pairs(D, None, box=box, bins=12, dmax=30.0)
        np.testing.assert_allclose(got, want, rtol=RTOL_W, atol=0)


def test_deferred_grid_builds(ctx):
    """PCF_OPT_GRID_DEFER: grids built back to back and completed by their
    first use (in another order than built) give the histograms of complete
    builds; an invalid catalog is reported by its first use and every later
    one."""
    from desi_b200.api import PCF_OPT_GRID_DEFER, PcfError
    box = 250.0
    cats = [catalog.neyman_scott(4000, box, seed=71), catalog.uniform(4100, box, seed=72),
            catalog.uniform(3900, box, seed=73, weights="uniform")]
    want = [ctx.count_pairs(ctx.grid(c, box), None, bins=20, dmax=60.0, ani="both", bpc=True)
            for c in cats]
    from desi_b200 import api
    c2 = api.Context(0)
    try:
        c2.set_option(PCF_OPT_GRID_DEFER, 1)
        gs = [c2.grid(c, box) for c in cats]
        for k in (2, 0, 1):
            got = c2.count_pairs(gs[k], None, bins=20, dmax=60.0, ani="both", bpc=True)
            for g_, w_ in zip(got, want[k]):
                np.testing.assert_allclose(g_, w_, rtol=1e-12, atol=0)
        dr = c2.count_pairs(gs[0], gs[1], bins=20, dmax=60.0, bpc=True)
        np.testing.assert_array_equal(dr, oracle.pairs(cats[0], cats[1], box=box, bins=20,
                                                        dmax=60.0, bpc=True))
        bad = cats[1].copy()
        bad[7, 0] = box + 1.0
        gb = c2.grid(bad, box)  # queued: the check comes with the first use
        for _ in range(2):
            with pytest.raises(PcfError):
                c2.count_pairs(gb, None, bins=20, dmax=60.0)
        with pytest.raises(PcfError):
            gb.info()
        gb.free()
        assert gs[2].info()["unit_weights"] is False
    finally:
        c2.close()


def _weighted(pts, rng, kind):
    out = pts.copy()
    n = len(out)
    if kind == "wide":      # log-uniform over three decades: no exact integer image, FP64 sums
        out[:, 3] = np.exp(rng.uniform(np.log(0.01), np.log(10.0), n)).astype(np.float32)
    elif kind == "zeros":   # a third of the weights exactly zero
        w = rng.uniform(0.5, 1.5, n).astype(np.float32)
        w[rng.random(n) < 0.33] = 0.0
        out[:, 3] = w
    elif kind == "signed":  # negative weights: FP64 shared sums
        out[:, 3] = rng.uniform(-1.0, 1.0, n).astype(np.float32)
    return out


@pytest.mark.parametrize("kind", ["wide", "zeros", "signed"])
@pytest.mark.parametrize("ani,bins", [(True, 30), (False, 100)])
def test_weighted_sum_paths(ctx, kind, ani, bins):
    """Weighted histograms through the fixed-point limb sums (zero weights)
    and the FP64 fallback (weights over three decades, negative weights),
    against the FP64 oracle.  The signed case is compared on |oracle| + 1 to keep the
    relative bound meaningful where positive and negative terms cancel."""
    rng = np.random.default_rng(17)
    box = 200.0
    D = _weighted(catalog.neyman_scott(2500, box, seed=21), rng, kind)
    R = _weighted(catalog.uniform(2600, box, seed=22), rng, kind)
    gd, gr = ctx.grid(D, box), ctx.grid(R, box)
    for bpc in (False, True):
        for (a, b, A, B) in ((gd, None, D, None), (gd, gr, D, R)):
            got = ctx.count_pairs(a, b, bins=bins, dmax=60.0, ani=ani, bpc=bpc)
            want = oracle.pairs(A, B, box=box, bins=bins, dmax=60.0, ani=ani, bpc=bpc)
            if kind == "signed":
                assert np.all(np.abs(got - want) <= RTOL_W * (np.abs(want) + 1.0))
            else:
                _cmp(got, want, True)


def test_weighted_dense_cells_flush_budget(ctx):
    """Tight clusters: a warp runs far more than 65536 pair tests, so the
    fixed-point copies flush mid-launch before a limb counter could wrap."""
    rng = np.random.default_rng(5)
    box = 100.0
    D = catalog.neyman_scott(12000, box, seed=31, children=2000, sigma=1.0, weights="uniform")
    g = ctx.grid(D, box)
    for ani in (False, True):
        got, st = ctx.count_pairs(g, None, bins=30, dmax=20.0, ani=ani, stats=True)
        want = oracle.pairs(D, None, box=box, bins=30, dmax=20.0, ani=ani)
        _cmp(got, want, True)
        assert st["candidates"] > 64 * 65536


def _tune_key(ani, bpc, cross, weighted, bins, n, box, dmax):
    """The library's tuning-table key of a pair-histogram class (tune.cu)."""
    import math
    nbar = n * 4.18879 * dmax ** 3 / box ** 3
    bucket = int(math.floor(2.0 * math.log2(nbar + 1.0) + 0.5))
    kind = "both" if ani == "both" else ("ani" if ani else "iso")
    return (f"{kind}{'-bpc' if bpc else ''}{'-xy' if cross else '-xx'}"
            f"{'-w' if weighted else '-u'}-b{bins}-n{bucket}")


@pytest.mark.parametrize("w", ["unit", "uniform"])
@pytest.mark.parametrize("ani", [False, True, "both"])
def test_every_histogram_scheme(tmp_path, w, ani):
    """Each shared-memory privatisation scheme (lane-private, per-warp, global,
    per-warp and lane-private fixed-point limbs), forced through a loaded
    tuning table, gives the oracle's histogram: bit-exact for unit weights,
    within 1e-12 for weights."""
    from desi_b200 import api
    box, bins, dmax, n = 250.0, 30, 80.0, 2500
    D = catalog.neyman_scott(n, box, seed=41, weights=w)
    R = catalog.uniform(n + 77, box, seed=42, weights=w)
    weighted = w != "unit"
    def ref(cross):
        kw = dict(box=box, bins=bins, dmax=dmax, bpc=True)
        B = R if cross else None
        if ani == "both":
            return np.concatenate([oracle.pairs(D, B, ani=False, **kw).ravel(),
                                   oracle.pairs(D, B, ani=True, **kw).ravel()])
        return oracle.pairs(D, B, ani=ani, **kw)
    want = {cross: ref(cross) for cross in (False, True)}
    for mode in (0, 1, 2, 3, 4):
        path = str(tmp_path / f"tune{mode}.txt")
        with open(path, "w") as f:
            for cross in (False, True):
                key = _tune_key(ani, True, cross, weighted, bins, n + 77 if cross else n, box, dmax)
                f.write(f"{key} 0 {mode} 1.0\n")
        c = api.Context(0)
        try:
            c.tune_load(path)
            gd, gr = c.grid(D, box), c.grid(R, box)
            for cross in (False, True):
                got = c.count_pairs(gd, gr if cross else None, bins=bins, dmax=dmax, ani=ani, bpc=True)
                if ani == "both":
                    got = np.concatenate([got[0].ravel(), got[1].ravel()])
                _cmp(got.ravel(), want[cross].ravel(), weighted)
        finally:
            c.close()


@pytest.mark.parametrize("w", ["unit", "uniform", "signed"])
@pytest.mark.parametrize("bpc", [False, True])
@pytest.mark.parametrize("bins", [30, 48])
def test_both_kinds(ctx, w, bpc, bins):
    """ani="both": the isotropic and anisotropic histograms equal the two
    single-kind calls (bit-exact for unit weights, 1e-12 for weights; the FP64
    fallback for signed weights) and the oracle.  Untuned, the call runs the
    two single-kind launches; the one-pass kernel (a tuned scheme) is covered
    by test_every_histogram_scheme."""
    rng = np.random.default_rng(23)
    box, dmax = 250.0, 80.0
    D = catalog.neyman_scott(2600, box, seed=51, weights="uniform" if w != "unit" else "unit")
    R = catalog.uniform(2700, box, seed=52, weights="uniform" if w != "unit" else "unit")
    if w == "signed":
        D = _weighted(D, rng, "signed")
        R = _weighted(R, rng, "signed")
    gd, gr = ctx.grid(D, box), ctx.grid(R, box)
    for (a, b, A, B) in ((gd, None, D, None), (gr, None, R, None), (gd, gr, D, R)):
        iso, ani = ctx.count_pairs(a, b, bins=bins, dmax=dmax, ani="both", bpc=bpc)
        for got, is_ani in ((iso, False), (ani, True)):
            single = ctx.count_pairs(a, b, bins=bins, dmax=dmax, ani=is_ani, bpc=bpc)
            want = oracle.pairs(A, B, box=box, bins=bins, dmax=dmax, ani=is_ani, bpc=bpc)
            if w == "signed":
                assert np.all(np.abs(got - want) <= RTOL_W * (np.abs(want) + 1.0))
                assert np.all(np.abs(got - single) <= RTOL_W * (np.abs(single) + 1.0))
            else:
                _cmp(got, want, w != "unit")
                _cmp(got, single, w != "unit")


@pytest.mark.parametrize("w", ["uniform", "signed"])
@pytest.mark.parametrize("bins", [30, 48])
def test_both_kinds_forced_one_pass(tmp_path, w, bins):
    """A both-kinds call tuned to one pass (exact weights: per-warp limbs with
    the isotropic copy in four sub-copies and the next candidate group loaded
    ahead; signed weights: per-warp FP64 sums) equals the two single-kind
    calls and the oracle (1e-12; the signed sums with an absolute floor)."""
    from desi_b200 import api
    rng = np.random.default_rng(29)
    box, dmax, n = 250.0, 80.0, 2400
    D = catalog.neyman_scott(n, box, seed=61, weights="uniform")
    R = catalog.uniform(n + 90, box, seed=62, weights="uniform")
    if w == "signed":
        D, R = _weighted(D, rng, "signed"), _weighted(R, rng, "signed")
    mode = 3 if w == "uniform" else 1
    path = str(tmp_path / "tune.txt")
    with open(path, "w") as f:
        for cross in (False, True):
            f.write(f"{_tune_key('both', True, cross, True, bins, n + 90 if cross else n, box, dmax)} 0 {mode} 1.0\n")
    c = api.Context(0)
    try:
        c.tune_load(path)
        gd, gr = c.grid(D, box), c.grid(R, box)
        for (a, b, A, B) in ((gd, None, D, None), (gd, gr, D, R)):
            (iso, ani), st = c.count_pairs(a, b, bins=bins, dmax=dmax, ani="both", bpc=True, stats=True)
            assert st["work_items"] > 0
            for got, is_ani in ((iso, False), (ani, True)):
                single = c.count_pairs(a, b, bins=bins, dmax=dmax, ani=is_ani, bpc=True)
                want = oracle.pairs(A, B, box=box, bins=bins, dmax=dmax, ani=is_ani, bpc=True)
                floor = 1.0 if w == "signed" else 0.0
                assert np.all(np.abs(got - want) <= RTOL_W * (np.abs(want) + floor))
                assert np.all(np.abs(got - single) <= RTOL_W * (np.abs(single) + floor))
    finally:
        c.close()


@pytest.mark.parametrize("tuned", [False, True])
def test_both_kinds_device_output(ctx, tmp_path, tuned):
    """ani="both" into a device buffer (bins + bins^2 doubles, isotropic
    first) equals the host-output call within 1e-12, as two launches
    (untuned) and as one pass (a tuned scheme)."""
    import torch
    from desi_b200 import api
    box, bins, dmax, n = 250.0, 30, 80.0, 2200
    D = catalog.neyman_scott(n, box, seed=71, weights="uniform")
    R = catalog.uniform(n + 40, box, seed=72, weights="uniform")
    c = api.Context(0)
    try:
        if tuned:
            path = str(tmp_path / "tune.txt")
            with open(path, "w") as f:
                for cross in (False, True):
                    f.write(f"{_tune_key('both', True, cross, True, bins, n + 40 if cross else n, box, dmax)} 0 3 1.0\n")
            c.tune_load(path)
        gd, gr = c.grid(D, box), c.grid(R, box)
        for b in (None, gr):
            iso, ani = c.count_pairs(gd, b, bins=bins, dmax=dmax, ani="both", bpc=True)
            out = torch.full((bins + bins * bins,), -1.0, dtype=torch.float64, device="cuda")
            c.count_pairs(gd, b, bins=bins, dmax=dmax, ani="both", bpc=True, out_device_ptr=out.data_ptr())
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            _cmp(got[:bins], iso, True)  # FP64 sums: atomic order varies, 1e-12
            _cmp(got[bins:], ani.ravel(), True)
    finally:
        c.close()


@pytest.mark.parametrize("variant", [1, 2])
@pytest.mark.parametrize("bpc", [False, True])
def test_one_pass_variants(tmp_path, variant, bpc):
    """The weighted one-pass kernel's variants (two isotropic sub-copies;
    plus candidates staged into shared memory) give the oracle's histograms
    within 1e-12, on catalogs dense enough for full 32-point tiles and on
    sparse ones (partial tiles take the unstaged path)."""
    from desi_b200 import api
    box, dmax, bins = 250.0, 80.0, 30
    for n in (2600, 9000):
        D = catalog.neyman_scott(n, box, seed=63, weights="uniform")
        R = catalog.uniform(n + 77, box, seed=64, weights="uniform")
        path = str(tmp_path / f"tune{n}.txt")
        with open(path, "w") as f:
            for cross in (False, True):
                f.write(f"{_tune_key('both', bpc, cross, True, bins, n + 77 if cross else n, box, dmax)} 0 3 1.0\n")
        c = api.Context(0)
        try:
            c.tune_load(path)
            c.set_option(api.PCF_OPT_PAIR_VARIANT, variant)
            gd, gr = c.grid(D, box), c.grid(R, box)
            for (a, b, A, B) in ((gd, None, D, None), (gd, gr, D, R)):
                iso, ani = c.count_pairs(a, b, bins=bins, dmax=dmax, ani="both", bpc=bpc)
                for got, is_ani in ((iso, False), (ani, True)):
                    want = oracle.pairs(A, B, box=box, bins=bins, dmax=dmax, ani=is_ani, bpc=bpc)
                    _cmp(got, want, True)
        finally:
            c.close()


@pytest.mark.parametrize("ani", [False, True, "both"])
@pytest.mark.parametrize("w", ["unit", "uniform"])
def test_half_tiles(tmp_path, ani, w):
    """Home tiles of 16 points (an autotuner candidate, forced through a
    loaded tuning table with the tile column) give the oracle's histograms."""
    from desi_b200 import api
    box, dmax, bins, n = 250.0, 80.0, 30, 3000
    D = catalog.neyman_scott(n, box, seed=65, weights=w)
    R = catalog.uniform(n + 50, box, seed=66, weights=w)
    path = str(tmp_path / "tune.txt")
    mode = 3 if (ani == "both" and w != "unit") else -1
    with open(path, "w") as f:
        for cross in (False, True):
            key = _tune_key(ani, True, cross, w != "unit", bins, n + 50 if cross else n, box, dmax)
            f.write(f"{key} 0 {mode} 1.0 16\n")
    c = api.Context(0)
    try:
        c.tune_load(path)
        gd, gr = c.grid(D, box), c.grid(R, box)
        for (a, b, A, B) in ((gd, None, D, None), (gd, gr, D, R)):
            got = c.count_pairs(a, b, bins=bins, dmax=dmax, ani=ani, bpc=True)
            kinds = ((got[0], False), (got[1], True)) if ani == "both" else ((got, ani),)
            for g, is_ani in kinds:
                want = oracle.pairs(A, B, box=box, bins=bins, dmax=dmax, ani=is_ani, bpc=True)
                _cmp(g, want, w != "unit")
    finally:
        c.close()
