"""GPU parity of the isotropic triplet histograms (DDD/RRR/DDR/DRR) against
the FP64 oracle.  Unit weights: bit-exact; weighted: rtol 1e-12."""
import os

import numpy as np
import pytest

import oracle
from desi_b200 import catalog
from desi_b200.api import PcfError

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _cmp(got, want, weighted):
    if weighted:
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=1e-9)
    else:
        assert np.array_equal(got, want), (np.abs(got - want).max(), int((got != want).sum()))


@pytest.mark.parametrize("bpc", [False, True])
@pytest.mark.parametrize("w", ["unit", "uniform"])
@pytest.mark.parametrize("clu", [False, True])
def test_triplets_small(ctx, bpc, w, clu):
    box, bins, dmax = 100.0, 12, 24.0
    gen = catalog.neyman_scott if clu else catalog.uniform
    D = gen(1200, box, seed=21, weights=w) if clu else gen(1200, box, seed=21, weights=w)
    R = catalog.uniform(1300, box, seed=22, weights=w)
    gd, gr = ctx.grid(D, box), ctx.grid(R, box)
    weighted = w != "unit"
    got = ctx.count_triplets(gd, bins=bins, dmax=dmax, bpc=bpc)
    _cmp(got, oracle.triplets_iso(D, box=box, bins=bins, dmax=dmax, bpc=bpc), weighted)
    got = ctx.count_triplets(gd, gr, bins=bins, dmax=dmax, bpc=bpc)
    _cmp(got, oracle.triplets_iso(D, R, box=box, bins=bins, dmax=dmax, bpc=bpc), weighted)
    got = ctx.count_triplets(gr, gd, bins=bins, dmax=dmax, bpc=bpc)
    _cmp(got, oracle.triplets_iso(R, D, box=box, bins=bins, dmax=dmax, bpc=bpc), weighted)


def test_triplets_lattice_edges(ctx):
    g = np.stack(np.meshgrid(np.arange(9), np.arange(9), np.arange(9), indexing="ij"), -1)
    pts = np.concatenate([g.reshape(-1, 3).astype(np.float32) * 2.0 + 0.5,
                          np.ones((9 ** 3, 1), np.float32)], 1)
    box = 18.0
    gp = ctx.grid(pts, box)
    for bpc in (False, True):
        for bins, dmax in ((6, 6.0), (4, 8.0)):
            got = ctx.count_triplets(gp, bins=bins, dmax=dmax, bpc=bpc)
            _cmp(got, oracle.triplets_iso(pts, box=box, bins=bins, dmax=dmax, bpc=bpc), False)


def test_triplets_duplicates(ctx):
    base = catalog.uniform(300, 50.0, seed=31)
    pts = np.concatenate([base, base[:40]])
    other = np.concatenate([base[50:90], catalog.uniform(200, 50.0, seed=32)])
    a, b = ctx.grid(pts, 50.0), ctx.grid(other, 50.0)
    for bpc in (False, True):
        _cmp(ctx.count_triplets(a, bins=8, dmax=12.0, bpc=bpc),
             oracle.triplets_iso(pts, box=50.0, bins=8, dmax=12.0, bpc=bpc), False)
        _cmp(ctx.count_triplets(a, b, bins=8, dmax=12.0, bpc=bpc),
             oracle.triplets_iso(pts, other, box=50.0, bins=8, dmax=12.0, bpc=bpc), False)


def test_golden_config_full_size(ctx, catalogs, golden_3iso):
    """The reference's shipped run (data.dat / rand0.dat, 32768 points, 30 bins,
    dmax 60, plain): bit-exact against the FP64 oracle's histograms, and within
    FP32 edge effects of the reference's own results/*.example."""
    f = np.load(os.path.join(GOLDEN, "golden_3iso_fp64.npz"))
    D, R = catalogs["data"], catalogs["rand0"]
    gd, gr = ctx.grid(D, 251.0), ctx.grid(R, 251.0)
    got = {
        "DDD": ctx.count_triplets(gd, bins=30, dmax=60.0),
        "RRR": ctx.count_triplets(gr, bins=30, dmax=60.0),
        "DDR": ctx.count_triplets(gd, gr, bins=30, dmax=60.0),
        "DRR": ctx.count_triplets(gr, gd, bins=30, dmax=60.0),
    }
    for k, v in got.items():
        assert np.array_equal(v, f[k].astype(np.float64)), k
        g = golden_3iso[k]
        # the reference computed d^2 in FP32: a triangle near a bin edge may
        # sit in the neighbouring bin; totals of in-range triangles agree to 1e-6
        assert abs(v.sum() - g.sum()) <= 1e-6 * g.sum(), k
        assert np.abs(v - g).sum() <= 1e-5 * g.sum(), k


@pytest.mark.parametrize("bpc", [False, True])
@pytest.mark.parametrize("w", ["unit", "uniform"])
def test_triplets_ani(ctx, bpc, w):
    """bins^5 anisotropic triplets: ordered triples anchored at point 1."""
    box, bins, dmax = 60.0, 6, 14.0
    D = catalog.neyman_scott(700, box, seed=81, children=16, sigma=3.0, weights=w)
    R = catalog.uniform(800, box, seed=82, weights=w)
    gd, gr = ctx.grid(D, box), ctx.grid(R, box)
    weighted = w != "unit"
    _cmp(ctx.count_triplets(gd, bins=bins, dmax=dmax, ani=True, bpc=bpc),
         oracle.triplets_ani(D, box=box, bins=bins, dmax=dmax, bpc=bpc), weighted)
    _cmp(ctx.count_triplets(gd, gr, bins=bins, dmax=dmax, ani=True, bpc=bpc),
         oracle.triplets_ani(D, R, box=box, bins=bins, dmax=dmax, bpc=bpc), weighted)


@pytest.mark.parametrize("bpc", [False, True], ids=["plain", "periodic"])
def test_triplets_ani_equal_reference_kernels(ctx, bpc):
    """The GPU 3ani histograms (DDD, RRR, DDR, DRR) equal the reference's own
    3ani CUDA kernels, plain and periodic, bin for bin (committed fixtures,
    tests/golden/make_golden_3ani.py).  Periodic: through
    PCF_REF_NODE_GATES on the fixture's node grid; the default count, every
    triangle in range once, is larger."""
    g = np.load(os.path.join(GOLDEN, "golden_3ani_bpc.npz" if bpc else "golden_3ani.npz"))
    box, bins, dmax, P = float(g["box"]), int(g["bins"]), float(g["dmax"]), int(g["partitions"])
    gd, gr = ctx.grid(g["D"], box, partitions=P), ctx.grid(g["R"], box, partitions=P)
    for name, x, y in (("DDD", gd, None), ("RRR", gr, None), ("DDR", gd, gr), ("DRR", gr, gd)):
        got = ctx.count_triplets(x, y, bins=bins, dmax=dmax, ani=True, bpc=bpc, ref_gates=bpc)
        assert np.array_equal(got, g[name]), name
        if bpc:
            full = ctx.count_triplets(x, y, bins=bins, dmax=dmax, ani=True, bpc=True)
            assert full.sum() > got.sum()


def _lattice(n, seed, box_half=30):
    rng = np.random.default_rng(seed)
    D = np.ones((n, 4), np.float32)
    R = np.ones((n, 4), np.float32)
    D[:, :3] = 2 * rng.integers(0, box_half, size=(n, 3))
    R[:, :3] = 2 * rng.integers(0, box_half, size=(n, 3)) + 1
    return D, R


@pytest.mark.parametrize("ani", [False, True], ids=["3iso", "3ani"])
@pytest.mark.parametrize("P,dmax,bins", [(3, 20.0, 6), (6, 20.0, 8), (7, 12.0, 6)])
def test_triplets_ref_gates_equal_oracle(ctx, ani, P, dmax, bins):
    """PCF_REF_NODE_GATES: the periodic 3iso and 3ani counts of the
    reference's CUDA kernels (3isoBPC_k.cuh:191,940, 3aniBPC_k.cuh:210,959)
    equal the oracle's restatement of their node gates (which the CPU suite
    pins to a host build of those kernels) in DDD, RRR, DDR and DRR."""
    D, R = _lattice(600, 40 + P)
    box = 60.0
    gd, gr = ctx.grid(D, box, partitions=P), ctx.grid(R, box, partitions=P)
    f = oracle.triplets_ani if ani else oracle.triplets_iso
    for x, y, cx, cy in ((gd, None, D, None), (gr, None, R, None), (gd, gr, D, R), (gr, gd, R, D)):
        got = ctx.count_triplets(x, y, bins=bins, dmax=dmax, ani=ani, bpc=True, ref_gates=True)
        want = f(cx, cy, box=box, bins=bins, dmax=dmax, bpc=True, ref_gates=P)
        assert np.array_equal(got, want)


@pytest.mark.parametrize("ani", [False, True], ids=["3iso", "3ani"])
def test_triplets_ref_gates_weighted_clustered(ctx, ani):
    """The gated counts off the lattice: clustered data, weights U(0.5, 1.5),
    the reference's default 35 nodes per side, against the oracle."""
    box, bins, dmax, P = 250.0, 6 if ani else 10, 40.0, 35
    D = catalog.neyman_scott(900, box, seed=77)
    D[:, 3] = np.random.default_rng(3).uniform(0.5, 1.5, len(D)).astype(np.float32)
    R = catalog.uniform(700, box, seed=78)
    gd, gr = ctx.grid(D, box, partitions=P), ctx.grid(R, box, partitions=P)
    f = oracle.triplets_ani if ani else oracle.triplets_iso
    for x, y, cx, cy in ((gd, None, D, None), (gd, gr, D, R)):
        got = ctx.count_triplets(x, y, bins=bins, dmax=dmax, ani=ani, bpc=True, ref_gates=True)
        _cmp(got, f(cx, cy, box=box, bins=bins, dmax=dmax, bpc=True, ref_gates=P), True)


def test_triplets_ref_gates_arguments(ctx):
    """The gates need periodic counts and the caller's node grid."""
    D, R = _lattice(200, 9)
    g0 = ctx.grid(D, 60.0)
    g6 = ctx.grid(D, 60.0, partitions=6)
    g5 = ctx.grid(R, 60.0, partitions=5)
    with pytest.raises(PcfError):
        ctx.count_triplets(g6, bins=6, dmax=20.0, ani=True, bpc=False, ref_gates=True)
    with pytest.raises(PcfError):
        ctx.count_triplets(g0, bins=6, dmax=20.0, bpc=True, ref_gates=True)
    with pytest.raises(PcfError):
        ctx.count_triplets(g6, g5, bins=6, dmax=20.0, ani=True, bpc=True, ref_gates=True)


def test_wide_histogram_through_grown_staging(ctx):
    """A 70^3 histogram (2.7 MB of doubles) is larger than a context's initial
    page-locked staging buffer: the buffer grows and the result still equals
    the oracle, and a pair histogram on the same context afterwards too."""
    box, bins, dmax = 100.0, 70, 30.0
    D = catalog.neyman_scott(700, box, seed=31)
    gd = ctx.grid(D, box)
    got = ctx.count_triplets(gd, bins=bins, dmax=dmax, bpc=True)
    _cmp(got, oracle.triplets_iso(D, box=box, bins=bins, dmax=dmax, bpc=True), False)
    got2 = ctx.count_pairs(gd, None, bins=30, dmax=dmax, bpc=True)
    assert np.array_equal(got2, oracle.pairs(D, None, box=box, bins=30, dmax=dmax, bpc=True))
