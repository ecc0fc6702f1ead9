"""GPU parity at the sizes the bench measures.

* The headline step exactly as bench.py times it: the same catalogs and
  seeds (32768 Neyman-Scott + 32768 uniform, box 250, w ~ U(0.5, 1.5), 30
  bins, dmax 80, periodic), the partition count, kinds-in-one-pass and
  schemes its tuner picks, device outputs.  All six histograms against the
  FP64 oracle: weighted sums within 1e-12 relative (a single pair binned
  differently would move a bin by ~1e-5 relative), the unit-weight variant
  bit for bit.  The one-pass both-kinds kernel (four isotropic sub-copies)
  is also forced at this size, whatever the tuner picks on the box.
* The batched configuration at full size: the 200k clustered data catalog
  in a box of 1000 against the smallest (50k) and largest (400k) random
  catalogs, 40 bins, dmax 120 (ds = floor(40/120 * 1e6)/1e6), weighted,
  iso and ani, per call and through one persistent batch launch.
"""
import numpy as np
import pytest

import bench
import oracle
from desi_b200 import api, catalog

pytestmark = pytest.mark.gpu


def _tune_key(ani, bpc, cross, weighted, bins, n, box, dmax):
    """The library's tuning-table key of a pair-histogram class (tune.cu)."""
    import math
    nbar = n * 4.18879 * dmax ** 3 / box ** 3
    bucket = int(math.floor(2.0 * math.log2(nbar + 1.0) + 0.5))
    kind = "both" if ani == "both" else ("ani" if ani else "iso")
    return (f"{kind}{'-bpc' if bpc else ''}{'-xy' if cross else '-xx'}"
            f"{'-w' if weighted else '-u'}-b{bins}-n{bucket}")


def _run_step(ctx, D, R, P, kinds):
    import torch
    W = bench.WORKLOAD
    dev = torch.device("cuda", 0)
    outs = torch.zeros((6, W["bins"] + W["bins"] ** 2), dtype=torch.float64, device=dev)
    Dt, Rt = torch.from_numpy(D).to(dev), torch.from_numpy(R).to(dev)
    torch.cuda.synchronize()
    gd = ctx.grid(None, W["box"], partitions=P, device_ptr=Dt.data_ptr(), n=len(D))
    gr = ctx.grid(None, W["box"], partitions=P, device_ptr=Rt.data_ptr(), n=len(R))
    bench.step_calls(ctx, gd, gr, kinds, [outs[k].data_ptr() for k in range(6)])
    ctx.synchronize()
    got = bench.step_results(outs, kinds)
    gd.free()
    gr.free()
    return got


@pytest.fixture(scope="module")
def headline_catalogs():
    D, R = bench.catalogs()
    return D, R, bench.oracle_step(D, R)


def test_headline_step_tuned(headline_catalogs):
    D, R, want = headline_catalogs
    ctx = api.Context(0)
    try:
        P, fused, tuned = bench.tune_step(ctx, D, R)
        kinds = ("both",) if fused else (False, True)
        got = _run_step(ctx, D, R, P, kinds)
    finally:
        ctx.close()
    mm = bench.mismatches(got, want)
    assert sum(mm.values()) == 0, (mm, P, fused, tuned)
    for k in want:
        assert want[k].sum() > 0
        np.testing.assert_allclose(got[k], want[k], rtol=1e-12, atol=0)


@pytest.mark.parametrize("variant", [0, 1, 2, 3])
def test_headline_step_forced_one_pass(headline_catalogs, tmp_path, variant):
    """Both kinds in one pass with per-warp fixed-point limbs (scheme 3) at
    the headline size, P = 12, in each kernel variant: the isotropic copy in
    four sub-copies (0), in two (1), two with the candidates staged into
    shared memory by cp.async (2), and four with the anisotropic copy shared
    by each warp pair (3, five CTAs per SM)."""
    D, R, want = headline_catalogs
    W = bench.WORKLOAD
    path = str(tmp_path / "tune.txt")
    with open(path, "w") as f:
        for cross in (False, True):
            f.write(f"{_tune_key('both', True, cross, True, W['bins'], 32768, W['box'], W['dmax'])}"
                    " 0 3 1.0\n")
    ctx = api.Context(0)
    try:
        ctx.tune_load(path)
        ctx.set_option(api.PCF_OPT_PAIR_VARIANT, variant)
        got = _run_step(ctx, D, R, 12, ("both",))
    finally:
        ctx.close()
    mm = bench.mismatches(got, want)
    assert sum(mm.values()) == 0, mm


def test_headline_step_unit_weights():
    D, R = bench.catalogs()
    D[:, 3] = 1.0
    R[:, 3] = 1.0
    want = bench.oracle_step(D, R)
    ctx = api.Context(0)
    try:
        P, fused, _ = bench.tune_step(ctx, D, R)
        got = _run_step(ctx, D, R, P, ("both",) if fused else (False, True))
        got_split = _run_step(ctx, D, R, P, (False, True))
    finally:
        ctx.close()
    for k in want:
        assert np.array_equal(got[k], want[k]), k
        assert np.array_equal(got_split[k], want[k]), k


@pytest.fixture(scope="module")
def batched_catalogs():
    box = 1000.0
    D = catalog.neyman_scott(200_000, box, seed=4001, weights="uniform")
    R_small = catalog.uniform(50_000, box, seed=4100, weights="uniform")
    R_large = catalog.uniform(400_000, box, seed=4101, weights="uniform")
    return box, D, [R_small, R_large]


@pytest.mark.parametrize("ani", [False, True])
def test_batched_config_full_size(batched_catalogs, ani):
    box, D, Rs = batched_catalogs
    bins, dmax = 40, 120.0
    kw = dict(box=box, bins=bins, dmax=dmax, ani=ani)
    want_dd = oracle.pairs(D, **kw)
    want_rr = [oracle.pairs(R, **kw) for R in Rs]
    want_dr = [oracle.pairs(D, R, **kw) for R in Rs]
    ctx = api.Context(0)
    try:
        gd = ctx.grid(D, box)
        grs = [ctx.grid(R, box) for R in Rs]
        (dd, rr, dr), st = ctx.batch_pairs(gd, grs, bins=bins, dmax=dmax, ani=ani, stats=True)
        assert st["pairs"] > 1e9
        cmp = lambda g, w: np.testing.assert_allclose(g, w, rtol=1e-12, atol=0)  # noqa: E731
        cmp(dd, want_dd)
        cmp(ctx.count_pairs(gd, None, bins=bins, dmax=dmax, ani=ani), want_dd)
        for i, g in enumerate(grs):
            cmp(rr[i], want_rr[i])
            cmp(dr[i], want_dr[i])
            cmp(ctx.count_pairs(g, None, bins=bins, dmax=dmax, ani=ani), want_rr[i])
            cmp(ctx.count_pairs(gd, g, bins=bins, dmax=dmax, ani=ani), want_dr[i])
    finally:
        ctx.close()
