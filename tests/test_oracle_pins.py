"""CPU: pin the FP64 oracle against the reference's own outputs.

* FP32-emulation mode of the oracle vs the reference's CPU engines
  (cpp/2PCF*/normal, compiled in place by oracle/Makefile): bit-exact.
* FP32-emulation mode (nvcc's contraction d2 = fma(dz,dz, fma(dx,dx, dy*dy)))
  vs the shipped results/*iso.example of the reference CUDA program: bit-exact.
* FP64 canonical vs FP32 modes: every difference is an edge pair.
"""
import os

import numpy as np
import pytest

import oracle

L1K = 250.0


def _ref(kind):
    try:
        return oracle.RefEngine(kind)
    except FileNotFoundError:
        pytest.skip(f"oracle/_ref/libref_{kind}.so not built")


@pytest.mark.parametrize("bins,dmax,sn", [(30, 80.0, 20.0), (20, 150.0, 25.0), (17, 33.3, 9.0)])
def test_ref_cpu_2iso_xx_xy_bitexact(catalogs, bins, dmax, sn):
    D, R = catalogs["data_1K"], catalogs["rand0_1K"]
    e = _ref("2iso")
    # the CPU engine counts coincident points and has no bin cap (2PCF.h:197)
    xx = e.xx(D, box=L1K, size_node=sn, bins=bins, dmax=dmax)
    o = oracle.pairs(D, box=L1K, bins=bins, dmax=dmax, rule=0, prec=oracle.REF32_NOFMA)
    assert np.array_equal(xx, o)
    xy = e.xy(D, R, box=L1K, size_node=sn, bins=bins, dmax=dmax)
    o = oracle.pairs(D, R, box=L1K, bins=bins, dmax=dmax, rule=0, prec=oracle.REF32_NOFMA)
    assert np.array_equal(xy, o)


def test_ref_cpu_2ani_bitexact(catalogs):
    D, R = catalogs["data_1K"], catalogs["rand0_1K"]
    e = _ref("2ani")
    xx = e.xx(D, box=L1K, size_node=20.0, bins=30, dmax=80.0)
    o = oracle.pairs(D, box=L1K, bins=30, dmax=80.0, ani=True, rule=0, prec=oracle.REF32_NOFMA)
    assert np.array_equal(xx, o)
    xy = e.xy(D, R, box=L1K, size_node=20.0, bins=30, dmax=80.0)
    o = oracle.pairs(D, R, box=L1K, bins=30, dmax=80.0, ani=True, rule=0,
                     prec=oracle.REF32_NOFMA)
    assert np.array_equal(xy, o)


def test_ref_cpu_thread_count_does_not_change_result(catalogs):
    D = catalogs["data_1K"]
    e = _ref("2iso")
    e.set_threads(2)
    a = e.xx(D, box=L1K, size_node=20.0, bins=30, dmax=80.0)
    e.set_threads(os.cpu_count() or 4)
    b = e.xx(D, box=L1K, size_node=20.0, bins=30, dmax=80.0)
    e.set_threads(2)
    assert np.array_equal(a, b)


@pytest.mark.slow
def test_golden_ddd_bitexact_fp32_emulation(catalogs, golden_3iso):
    """results/DDDiso.example == oracle in the reference kernel's FP32 rounding."""
    h = oracle.triplets_iso(catalogs["data"], box=251.0, bins=30, dmax=60.0,
                            prec=oracle.REF32_FMA_B)
    assert np.array_equal(h, golden_3iso["DDD"])


@pytest.mark.slow
@pytest.mark.parametrize("name,x,y", [("DDR", "data", "rand0"), ("DRR", "rand0", "data")])
def test_golden_mixed_bitexact_fp32_emulation(catalogs, golden_3iso, name, x, y):
    h = oracle.triplets_iso(catalogs[x], catalogs[y], box=251.0, bins=30, dmax=60.0,
                            prec=oracle.REF32_FMA_B)
    assert np.array_equal(h, golden_3iso[name])


@pytest.mark.slow
def test_golden_rrr_bitexact_fp32_emulation(catalogs, golden_3iso):
    h = oracle.triplets_iso(catalogs["rand0"], box=251.0, bins=30, dmax=60.0,
                            prec=oracle.REF32_FMA_B)
    assert np.array_equal(h, golden_3iso["RRR"])


def test_fp64_vs_fp32_differ_only_near_edges(catalogs):
    """Every pair whose FP64 and FP32 bins differ lies within FP32 rounding
    of a bin edge or of dmax."""
    D = catalogs["data_1K"][:600]
    bins, dmax = 30, 80.0
    ds = oracle.ds(bins, dmax)
    p = D[:, :3].astype(np.float64)
    d2 = ((p[:, None, :] - p[None, :, :]) ** 2).sum(-1)
    f = D[:, :3]
    dxf = (f[None, :, :] - f[:, None, :]).astype(np.float32)
    d2f = np.float32(dxf[..., 2] * dxf[..., 2] + (dxf[..., 0] * dxf[..., 0] + dxf[..., 1] * dxf[..., 1]))
    i, j = np.triu_indices(len(D), 1)
    r64 = np.sqrt(d2[i, j]) * ds
    r32 = np.sqrt(d2f[i, j].astype(np.float64)) * ds
    b64 = np.where(d2[i, j] < dmax * dmax, np.floor(r64), -1)
    b32 = np.where(d2f[i, j].astype(np.float64) < dmax * dmax, np.floor(r32), -1)
    diff = b64 != b32
    if diff.any():
        frac = r64[diff] - np.floor(r64[diff])
        near = np.minimum(frac, 1 - frac) < 1e-5 * bins
        assert near.all()


# ---------------------------------------------------------------------------
# Periodic (BPC), weighted and analytic rules against the reference's CPU
# engines, compiled in place by oracle/Makefile.
# ---------------------------------------------------------------------------

def _cat(kind, n, seed, weights="unit", box=250.0):
    from desi_b200 import catalog
    f = catalog.neyman_scott if kind == "clustered" else catalog.uniform
    return f(n, box, seed=seed, weights=weights)


@pytest.mark.parametrize("bins,dmax,sn", [(30, 80.0, 20.0), (20, 100.0, 25.0), (17, 33.3, 9.0)])
@pytest.mark.parametrize("kind", ["2iso_bpc", "2ani_bpc"])
def test_ref_cpu_bpc_bitexact(catalogs, kind, bins, dmax, sn):
    """The oracle's emulation of the periodic CPU engines (FP32 distances,
    <= for direct and < for image pairs, FP32 weight products) equals
    cpp/2PCF{isotropic,anisotropic}/BPC bit for bit."""
    D, R = catalogs["data_1K"], catalogs["rand0_1K"]
    e = _ref(kind)
    ani = kind.startswith("2ani")
    kw = dict(box=L1K, bins=bins, dmax=dmax, ani=ani, bpc=True, prec=oracle.REF32_CPU_BPC)
    assert np.array_equal(e.xx(D, box=L1K, size_node=sn, bins=bins, dmax=dmax),
                          oracle.pairs(D, **kw))
    assert np.array_equal(e.xy(D, R, box=L1K, size_node=sn, bins=bins, dmax=dmax),
                          oracle.pairs(D, R, **kw))


@pytest.mark.parametrize("kind", ["2iso_bpc", "2ani_bpc"])
def test_ref_cpu_bpc_weighted(kind):
    """Weighted clustered catalogs (w ~ U(0.5, 1.5)) at 8192 points: the
    compensated oracle sums match the engines' FP64 sums to 1e-12."""
    e = _ref(kind)
    e.set_threads(os.cpu_count() or 4)
    D = _cat("clustered", 8192, 11, "uniform")
    R = _cat("uniform", 8192, 12, "uniform")
    sn = 2.176 * 250.0 / 8192 ** (1 / 3)
    kw = dict(box=250.0, bins=30, dmax=80.0, ani=kind.startswith("2ani"), bpc=True,
              prec=oracle.REF32_CPU_BPC)
    for got, want in ((e.xx(D, box=250.0, size_node=sn, bins=30, dmax=80.0), oracle.pairs(D, **kw)),
                      (e.xy(D, R, box=250.0, size_node=sn, bins=30, dmax=80.0),
                       oracle.pairs(D, R, **kw))):
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=0)
        assert want.sum() > 0


def test_fp64_vs_cpu_bpc_differ_only_near_edges():
    """Every pair that the canonical FP64 rule and the emulated CPU periodic
    engine bin differently lies within FP32 rounding of a bin edge or of
    dmax (minimum image per axis)."""
    D = _cat("clustered", 900, 21)
    bins, dmax, L = 30, 80.0, 250.0
    ds = oracle.ds(bins, dmax)
    p = D[:, :3].astype(np.float64)
    i, j = np.triu_indices(len(D), 1)
    d = p[j] - p[i]
    d = np.where(d > L / 2, d - L, np.where(d < -L / 2, d + L, d))
    d2 = (d[:, 0] ** 2 + d[:, 1] ** 2) + d[:, 2] ** 2
    f = (D[i, :3] - D[j, :3]).astype(np.float32)
    wrapped = np.abs(f) > np.float32(L / 2)
    f = np.where(wrapped, np.abs(f) - np.float32(L), f).astype(np.float32)
    d2f = ((f[:, 0] * f[:, 0] + f[:, 1] * f[:, 1]) + f[:, 2] * f[:, 2]).astype(np.float64)
    dd = float(np.float32(dmax) * np.float32(dmax))
    in64 = (d2 > 0) & (d2 < dd)
    in32 = np.where(wrapped.any(1), d2f < dd, d2f <= dd)
    b64 = np.where(in64, np.floor(np.sqrt(d2) * ds), -1)
    b32 = np.where(in32, np.floor(np.sqrt(d2f) * ds), -1)
    diff = b64 != b32
    r = np.sqrt(d2[diff]) * ds
    near_edge = np.minimum(r - np.floor(r), np.ceil(r) - r) < 1e-5 * bins
    near_dmax = np.abs(np.sqrt(d2[diff]) - dmax) < 1e-4
    zero = d2[diff] == 0
    assert (near_edge | near_dmax | zero).all()
    # and the histograms differ only by those pairs
    h64 = oracle.pairs(D, box=L, bins=bins, dmax=dmax, bpc=True, rule=oracle.RULE_EXCL_ZERO)
    h32 = oracle.pairs(D, box=L, bins=bins, dmax=dmax, bpc=True, prec=oracle.REF32_CPU_BPC)
    # (each such XX pair moves 2 counts out of one bin and at most into another)
    assert np.abs(h64 - h32).sum() <= 4 * diff.sum()


def test_oracle_cells_equal_brute():
    """The cell-pruned oracle (used for the large parity cases) gives the
    brute-force histogram: counts bit for bit, weighted sums to 1e-15."""
    box = 1000.0
    D = _cat("clustered", 12000, 31, "uniform", box=box)
    R = _cat("uniform", 15000, 32, "uniform", box=box)
    for ani in (False, True):
        for bpc in (False, True):
            for B in (None, R):
                kw = dict(box=box, bins=40, dmax=120.0, ani=ani, bpc=bpc)
                a = oracle.pairs(D, B, method="brute", **kw)
                b = oracle.pairs(D, B, method="cells", **kw)
                np.testing.assert_allclose(b, a, rtol=1e-15, atol=0)
                Du = D.copy(); Du[:, 3] = 1
                Bu = None if B is None else B.copy()
                if Bu is not None:
                    Bu[:, 3] = 1
                assert np.array_equal(oracle.pairs(Du, Bu, method="brute", **kw),
                                      oracle.pairs(Du, Bu, method="cells", **kw))


def _ref_analytic():
    try:
        return oracle.RefAnalyticRR()
    except FileNotFoundError:
        pytest.skip("oracle/_ref/libref_2iso_analytic.so not built")


def _ref_3iso():
    try:
        return oracle.Ref3IsoBPC()
    except FileNotFoundError:
        pytest.skip("oracle/_ref/libref_3iso_bpc.so not built")


def _cpu_rr(n, L, dmax, nbins, dr_f32):
    """The CPU engines' analytic RR (cpp/2PCFisotropic/BPC_analitic/2PCF.h:333-355,
    cpp/3PCFisotropic/BPC/3PCFiso.h:1794-1812): beta = n/L * (float)(n/L) / L
    in FP64, alpha = 4 pi beta dr^3 / 3, RR[a] = alpha ((a+1)^3 - a^3), with
    dr = d_max/bn in FP32 (2-point engine) or in FP64 (3-point engine)."""
    f32 = np.float32
    dr = np.float64(f32(dmax) / f32(nbins)) if dr_f32 else np.float64(f32(dmax)) / nbins
    beta = n / np.float64(L)
    beta *= np.float64(f32(n) / f32(L))
    beta /= np.float64(L)
    alph = 4 * (2 * np.arccos(0.0)) * beta / 3
    alph *= dr * dr * dr
    r2 = np.arange(nbins, dtype=np.float64)
    r1 = r2 + 1
    return alph * ((r1 * r1 * r1) - (r2 * r2 * r2))


@pytest.mark.parametrize("bins,dmax", [(30, 80.0), (20, 100.0), (17, 33.3)])
def test_ref_analytic_rr(bins, dmax):
    """cpp/2PCFisotropic/BPC_analitic: its periodic DD equals the oracle's CPU
    emulation bit for bit, its RR the restated CPU formula, and the oracle's
    analytic RR (the CUDA path's constants, pcf2isoBPC.cuh:199-202, which
    round N^2/L^3 to FP32) agrees with it to the FP32 rounding of beta."""
    e = _ref_analytic()
    D = _cat("uniform", 4096, 5)
    sn = 2.276 * 250.0 / 4096 ** (1 / 3)
    dd, rr = e.dd_rr(D, box=250.0, size_node=sn, bins=bins, dmax=dmax)
    assert np.array_equal(dd, oracle.pairs(D, box=250.0, bins=bins, dmax=dmax, bpc=True,
                                           prec=oracle.REF32_CPU_BPC))
    np.testing.assert_allclose(rr, _cpu_rr(len(D), 250.0, dmax, bins, True), rtol=1e-15, atol=0)
    a = oracle.analytic_rr(bins, len(D), 250.0, dmax, wrap=False)
    np.testing.assert_allclose(a, rr, rtol=1.2e-7, atol=0)


@pytest.mark.parametrize("n,dmax,kind,seed", [(2048, 60.0, "uniform", 7),
                                              (4096, 80.0, "clustered", 7),
                                              (8192, 50.0, "clustered", 8)])
def test_ref_3iso_bpc_ddd_bitexact(n, dmax, kind, seed):
    """cpp/3PCFisotropic/BPC (NODE3P, its own node-image passes, FP32
    distances, float symmetrisation) gives the oracle's FP64 periodic DDD
    (consistent embedding) bit for bit on these catalogs.  (Larger or denser
    catalogs hold pairs within FP32 rounding of a bin edge, which move every
    triangle they belong to between adjacent cells, totals unchanged.)"""
    e = _ref_3iso()
    e.set_threads(os.cpu_count() or 4)
    D = _cat(kind, n, seed)
    sn = 2.17 * 250.0 / n ** (1 / 3)
    h = e.xxx(D, box=250.0, size_node=sn, bins=30, dmax=dmax)
    o = oracle.triplets_iso(D, box=250.0, bins=30, dmax=dmax, bpc=True)
    assert o.sum() > 0
    assert np.array_equal(h, o)


def test_ref_3iso_analytic_ff_ref(tmp_path):
    """The analytic 3iso path of cpp/3PCFisotropic/BPC (make_histo_analitic,
    3PCFiso.h:1484): the oracle's make_ff_av_ref on the engine's own fine DD
    (600 000 bins) and RR reproduces the engine's ff_av_ref.dat (written
    with 12 significant digits).  The fine DD itself agrees with the oracle's
    FP32 emulation up to the engine's own fault: its Z-only image pass reads
    dis_nod, which that loop never sets (3PCFiso.h:1794; the value left by an
    earlier loop or the stack), and so now and then skips a node pair's image
    pass, dropping a few dozen pairs.  So the engine never has more pairs
    than the emulation in any bin and misses at most 0.1% of them.  (Its
    RRR/DDR refinement loop is commented out, 3PCFiso.h:1623-1710, so the
    CUDA kernels are the only reference for the refined histograms.)"""
    e = _ref_3iso()
    e.set_threads(os.cpu_count() or 4)
    D = _cat("uniform", 2048, 9)
    bins, dmax = 30, 80.0
    sn = 2.17 * 250.0 / 2048 ** (1 / 3)
    ff, ffr, dd = e.analytic_ff(D, box=250.0, size_node=sn, bins=bins, dmax=dmax,
                                workdir=str(tmp_path))
    nref = 100 * 200 * bins
    dsf = float(np.float32(np.float32(nref) / np.float32(dmax)))
    emu = oracle.pairs(D, box=250.0, bins=nref, dmax=dmax, bpc=True, prec=oracle.REF32_CPU_BPC,
                       rule=0, ds_value=dsf)
    assert np.all(dd <= emu)
    assert emu.sum() - dd.sum() <= 1e-3 * emu.sum()
    got = oracle.ff_average_ref(dd, _cpu_rr(len(D), 250.0, dmax, nref, False), bins=bins,
                                dmax=dmax)
    np.testing.assert_allclose(got, ffr, rtol=1e-10, atol=1e-10)


@pytest.mark.parametrize("bpc", [False, True], ids=["plain", "periodic"])
def test_oracle_3ani_matches_reference_kernels(bpc):
    """The anisotropic 3-point oracle against the reference's own 3ani CUDA
    kernels, all bn^5 bins of DDD, RRR, DDR and DRR, from the committed
    fixtures (tests/golden/make_golden_3ani.py): plain XXX3ani / XXY3ani
    (cuda/kernels/3ani_k.cuh:8,109) and periodic XXX3ani_BPC / XXY3ani_BPC
    (cuda/kernels/3aniBPC_k.cuh:210,959, whose angle takes dz = |dz| - box
    for a pair joined through its z image, and which count through the
    reference's node gates: the oracle's ref_gates mode on the fixture's
    node grid).  Bit-equal counts."""
    name_ = "golden_3ani_bpc.npz" if bpc else "golden_3ani.npz"
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", name_))
    kw = dict(box=float(g["box"]), bins=int(g["bins"]), dmax=float(g["dmax"]), bpc=bpc,
              ref_gates=int(g["partitions"]) if bpc else 0)
    D, R = g["D"], g["R"]
    for name, x, y in (("DDD", D, None), ("RRR", R, None), ("DDR", D, R), ("DRR", R, D)):
        got = oracle.triplets_ani(x, y, **kw)
        want = g[name]
        assert want.sum() > 1e6
        assert np.array_equal(got, want), (name, float(np.abs(got - want).sum()))


def _host_kernels():
    if not oracle.ref_kernels_available():
        pytest.skip("oracle/_ref/libref_kernels_host.so not built")
    return oracle.ref_kernels_3pt


def _lattice(n, seed):
    """Data on even, randoms on odd integer coordinates of a 60-box: every
    FP32 sum the reference's kernels form is exact."""
    rng = np.random.default_rng(seed)
    D = np.ones((n, 4), np.float32)
    R = np.ones((n, 4), np.float32)
    D[:, :3] = 2 * rng.integers(0, 30, size=(n, 3))
    R[:, :3] = 2 * rng.integers(0, 30, size=(n, 3)) + 1
    return D, R


@pytest.mark.parametrize("bpc", [False, True], ids=["plain", "periodic"])
def test_host_build_of_reference_kernels_equals_b200_run(bpc):
    """The reference's 3ani kernels compiled for the host
    (oracle/ref_kernels_host.cpp) give the B200 run of the same kernels
    (tests/golden/golden_3ani*.npz) bin for bin: the host build is a pin at
    any configuration, not only at the fixture's."""
    ref = _host_kernels()
    g = np.load(os.path.join(os.path.dirname(__file__), "golden",
                             "golden_3ani_bpc.npz" if bpc else "golden_3ani.npz"))
    h = ref(g["D"], g["R"], ani=True, bpc=bpc, box=float(g["box"]), bins=int(g["bins"]),
            dmax=float(g["dmax"]), partitions=int(g["partitions"]))
    for name in ("DDD", "RRR", "DDR", "DRR"):
        assert np.array_equal(h[name], g[name]), name


@pytest.mark.parametrize("ani", [False, True], ids=["3iso", "3ani"])
@pytest.mark.parametrize("P,dmax,bins,n", [(6, 20.0, 8, 700), (3, 20.0, 6, 300), (4, 18.0, 5, 400),
                                           (7, 12.0, 6, 500), (2, 16.0, 5, 200)])
def test_oracle_reference_gates_equal_reference_kernels(ani, P, dmax, bins, n):
    """Periodic triplets: the reference's CUDA kernels (XXX3iso_BPC /
    XXY3iso_BPC, 3isoBPC_k.cuh:191,940; XXX3ani_BPC / XXY3ani_BPC,
    3aniBPC_k.cuh:210,959) count a triangle once per node-gate block that
    passes.  The oracle's ref_gates mode (the 64 blocks as a table, with the
    reference's defective gates) equals them in DDD, RRR, DDR and DRR on
    coarse and fine node grids; the nearest-image count (the default, which
    the reference's CPU engine follows) is larger wherever a defective gate
    drops triangles."""
    ref = _host_kernels()
    D, R = _lattice(n, 100 + P)
    L = 60.0
    h = ref(D, R, ani=ani, bpc=True, box=L, bins=bins, dmax=dmax, partitions=P)
    f = oracle.triplets_ani if ani else oracle.triplets_iso
    for name, x, y in (("DDD", D, None), ("RRR", R, None), ("DDR", D, R), ("DRR", R, D)):
        got = f(x, y, box=L, bins=bins, dmax=dmax, bpc=True, ref_gates=P)
        assert np.array_equal(got, h[name]), name
        full = f(x, y, box=L, bins=bins, dmax=dmax, bpc=True)
        assert full.sum() >= got.sum()


@pytest.mark.parametrize("ani", [False, True], ids=["3iso", "3ani"])
@pytest.mark.parametrize("P,dmax,bins", [(6, 20.0, 8), (3, 25.0, 6), (10, 12.0, 5)])
def test_oracle_plain_3pt_equals_reference_kernels(ani, P, dmax, bins):
    """Without periodic boundaries the reference's 3-point kernels (XXX3iso /
    XXY3iso, 3iso_k.cuh:8,94; XXX3ani / XXY3ani, 3ani_k.cuh:8,109) have no
    node gates to get wrong: on any node grid they equal the oracle's default
    rule."""
    ref = _host_kernels()
    D, R = _lattice(800, 5 + P)
    L = 60.0
    h = ref(D, R, ani=ani, bpc=False, box=L, bins=bins, dmax=dmax, partitions=P)
    f = oracle.triplets_ani if ani else oracle.triplets_iso
    for name, x, y in (("DDD", D, None), ("RRR", R, None), ("DDR", D, R), ("DRR", R, D)):
        assert np.array_equal(f(x, y, box=L, bins=bins, dmax=dmax), h[name]), name


@pytest.mark.parametrize("bpc", [False, True], ids=["plain", "periodic"])
@pytest.mark.parametrize("P,dmax,bins", [(6, 20.0, 8), (3, 20.0, 6), (7, 12.0, 6), (35, 20.0, 10)])
def test_oracle_pairs_equal_reference_kernels(bpc, P, dmax, bins):
    """The pair rules of the headline step against the reference's own CUDA
    pair kernels compiled for the host (XX2iso / XY2iso, 2iso_k.cuh:8,63;
    XX2iso_BPC / XY2iso_BPC, 2isoBPC_k.cuh:8,284; XX2ani, 2ani_k.cuh:7;
    XX2ani_BPC, 2aniBPC_k.cuh:8) on lattice catalogs and node grids of 3 to
    35 per side: DD, RR and DR (iso), DD and RR (ani) bit-equal.  The
    anisotropic cross kernels read an out-of-range (XY2ani) or unset
    (XY2ani_BPC) weight; the anisotropic DR is pinned to the reference's CPU
    engines instead (test_ref_cpu_bpc_bitexact, test_ref_cpu_bpc_weighted)."""
    if not oracle.ref_kernels_available():
        pytest.skip("oracle/_ref/libref_kernels_host.so not built")
    D, R = _lattice(2500, 200 + P)
    L = 60.0
    for ani in (False, True):
        h = oracle.ref_kernels_2pt(D, R, ani=ani, bpc=bpc, box=L, bins=bins, dmax=dmax, partitions=P)
        kw = dict(box=L, bins=bins, dmax=dmax, bpc=bpc, ani=ani, ds_exact=bpc and not ani)
        assert np.array_equal(h["DD"], oracle.pairs(D, None, **kw)), ("DD", ani)
        assert np.array_equal(h["RR"], oracle.pairs(R, None, **kw)), ("RR", ani)
        if not ani:
            assert np.array_equal(h["DR"], oracle.pairs(D, R, **kw)), "DR"
        else:
            assert np.isnan(h["DR"]).all()
