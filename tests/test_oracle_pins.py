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
