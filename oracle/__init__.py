"""CPU checkers for the pair / triplet counting library.

TEST INFRASTRUCTURE ONLY.  Only ``tests/``, ``__graft_entry__.smoke()`` and
the CPU-baseline leg of ``bench.py`` import this package, and only as the
checker: the shipped library (``desi_b200``) never calls into it.

* :func:`pairs`, :func:`triplets_iso`, :func:`triplets_ani`,
  :func:`analytic_rr`, :func:`analytic_3iso` wrap ``liboracle.so``, our FP64
  restatement of the reference's histogram rules (``pcf_oracle.c`` cites the
  reference file:line each rule follows).
* :class:`RefEngine` wraps ``_ref/libref_*.so``: the reference's own CPU
  OpenMP engines (``cpp/2PCF*/{normal,BPC}``) compiled in place by
  ``oracle/Makefile``; used to pin the restatement and as the timed CPU
  baseline.
* :func:`ref_kernels_2pt`, :func:`ref_kernels_3pt` wrap
  ``_ref/libref_kernels_host.so``: the reference's CUDA pair and triplet
  kernels compiled unmodified for the host (``ref_kernels_host.cpp``).
* :func:`ref_read_catalog`, :func:`ref_save_histogram` wrap the reference's
  reader and writers (``_ref/libref_io.so``); ``ref_cuda`` runs the
  reference's CUDA program.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(HERE, "liboracle.so")

FP64, REF32_NOFMA, REF32_FMA_A, REF32_FMA_B, REF32_FMA_C = 0, 1, 2, 3, 4
# the reference's CPU periodic engines (cpp/2PCF{isotropic,anisotropic}/BPC),
# FP32 throughout; see cpu_bpc_slot in pcf_oracle.c
REF32_CPU_BPC = 5
_METHODS = {"auto": 0, "brute": 1, "cells": 2}
RULE_EXCL_ZERO, RULE_INCLUSIVE = 1, 2

_dptr = ctypes.POINTER(ctypes.c_double)
_fptr = ctypes.c_void_p


def build() -> None:
    """Compile liboracle.so (and _ref/ when the reference tree is present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def _load():
    if not os.path.exists(_LIB):
        build()
    lib = ctypes.CDLL(_LIB)
    lib.orc_pairs.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_uint,
                              ctypes.c_int, ctypes.c_double, ctypes.c_int,
                              _fptr, ctypes.c_long, _fptr, ctypes.c_long, ctypes.c_float,
                              ctypes.c_int, ctypes.c_float, _dptr]
    lib.orc_pairs_m.argtypes = lib.orc_pairs.argtypes + [ctypes.c_int]
    lib.orc_triplets_iso.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _fptr,
                                     ctypes.c_long, _fptr, ctypes.c_long, ctypes.c_float,
                                     ctypes.c_int, ctypes.c_float, ctypes.c_int, _dptr]
    lib.orc_triplets_ani.argtypes = [ctypes.c_int, ctypes.c_int, _fptr, ctypes.c_long,
                                     _fptr, ctypes.c_long, ctypes.c_float, ctypes.c_int,
                                     ctypes.c_float, ctypes.c_int, _dptr]
    lib.orc_analytic_rr.argtypes = [ctypes.c_int, ctypes.c_long, ctypes.c_float,
                                    ctypes.c_float, ctypes.c_int, _dptr]
    lib.orc_analytic_3iso.argtypes = [_fptr, ctypes.c_long, ctypes.c_float, ctypes.c_int,
                                      ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      _dptr, _dptr, _dptr, _dptr]
    lib.orc_analytic_ff.argtypes = [_fptr, ctypes.c_long, ctypes.c_float, ctypes.c_int,
                                    ctypes.c_float, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    _dptr, _dptr, _dptr]
    lib.orc_analytic_bin.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                     ctypes.c_float, ctypes.c_int, ctypes.c_double, _dptr,
                                     _dptr, _dptr]
    lib.orc_ff_average_ref.argtypes = [_dptr, _dptr, ctypes.c_int, ctypes.c_float,
                                       ctypes.c_int, ctypes.c_int, _dptr]
    lib.orc_ds.argtypes = [ctypes.c_int, ctypes.c_float, ctypes.c_int]
    lib.orc_ds.restype = ctypes.c_double
    return lib


_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = _load()
    return _lib


def _pts(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    assert a.ndim == 2 and a.shape[1] == 4
    return a


def _p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def _d(a):
    return a.ctypes.data_as(_dptr)


def ds(bins: int, dmax: float, exact: bool = False) -> float:
    return lib().orc_ds(bins, dmax, 1 if exact else 0)


def pairs(A, B=None, *, box: float, bins: int, dmax: float, ani: bool = False,
          bpc: bool = False, rule: int | None = None, ds_exact: bool = False,
          ds_value: float = 0.0, prec: int = FP64, method: str = "auto") -> np.ndarray:
    """Pair histogram.  ``B is None`` -> XX over A (ordered pairs), else XY.

    ``rule`` defaults to the reference CUDA rule for the variant (see
    :func:`reference_rule`).  ``method``: "brute" tests every pair, "cells"
    only pairs of adjacent cells of side >= dmax (same histogram), "auto"
    picks "cells" for large inputs.  Weighted sums are compensated, so they
    carry about one rounding of the total whatever the order of additions.
    """
    A = _pts(A)
    self_ = B is None
    Bp = A if self_ else _pts(B)
    if rule is None:
        # the CPU periodic engines count direct pairs with <= (2PCF.h:199)
        rule = (RULE_INCLUSIVE if prec == REF32_CPU_BPC
                else reference_rule(ani=ani, bpc=bpc, cross=not self_))
    nb = bins * bins if ani else bins
    out = np.zeros(nb, np.float64)
    rc = lib().orc_pairs_m(int(ani), int(bpc), int(self_), rule, int(ds_exact), float(ds_value),
                           prec, _p(A), len(A), _p(Bp), len(Bp), box, bins, dmax, _d(out),
                           _METHODS[method])
    assert rc == 0
    return out.reshape(bins, bins) if ani else out


def reference_rule(*, ani: bool, bpc: bool, cross: bool) -> int:
    """Rule flags of the reference CUDA kernel for one pair variant.

    2iso  XX: d>0            (2iso_k.cuh:50)      XY: none   (2iso_k.cuh:107)
    2isoB XX: d>0            (2isoBPC_k.cuh:62)   XY: none   (2isoBPC_k.cuh:338)
    2ani  XX,XY: every component >0 (2ani_k.cuh:52,121)
    2aniB XX: >0 and <=      (2aniBPC_k.cuh:63)   XY: <= only (2aniBPC_k.cuh:401)
    """
    if not ani:
        return 0 if cross else RULE_EXCL_ZERO
    if not bpc:
        return RULE_EXCL_ZERO
    return RULE_INCLUSIVE if cross else (RULE_INCLUSIVE | RULE_EXCL_ZERO)


def triplets_iso(X, Y=None, *, box: float, bins: int, dmax: float, bpc: bool = False,
                 prec: int = FP64, ref_gates: int = 0):
    """ref_gates > 0 (periodic only): count each ordered triangle as often as
    the reference's periodic CUDA node gates do on a grid of ref_gates nodes
    per side (3isoBPC_k.cuh:191,940), its gate defects included."""
    X = _pts(X)
    mixed = Y is not None
    Yp = _pts(Y) if mixed else X
    out = np.zeros(bins ** 3, np.float64)
    rc = lib().orc_triplets_iso(int(bpc), int(mixed), prec, _p(X), len(X), _p(Yp), len(Yp),
                                box, bins, dmax, int(ref_gates), _d(out))
    assert rc == 0
    return out.reshape(bins, bins, bins)


def triplets_ani(X, Y=None, *, box: float, bins: int, dmax: float, bpc: bool = False,
                 ref_gates: int = 0):
    """ref_gates > 0 (periodic only): count each ordered triangle as often as
    the reference's periodic node gates do on a grid of ref_gates nodes per
    side (3aniBPC_k.cuh:210,959), its gate defects included."""
    X = _pts(X)
    mixed = Y is not None
    Yp = _pts(Y) if mixed else X
    out = np.zeros(bins ** 5, np.float64)
    rc = lib().orc_triplets_ani(int(bpc), int(mixed), _p(X), len(X), _p(Yp), len(Yp), box,
                                bins, dmax, int(ref_gates), _d(out))
    assert rc == 0
    return out.reshape((bins,) * 5)


def analytic_rr(bins: int, n: int, box: float, dmax: float, wrap: bool = True):
    out = np.zeros(bins, np.float64)
    lib().orc_analytic_rr(bins, n, box, dmax, int(wrap), _d(out))
    return out


def analytic_3iso(D, *, box: float, bins: int, dmax: float, ptt: int = 100,
                  bn_ref: int = 200, wrap: bool = True):
    """Returns (DDR, RRR, ff_av, ff_av_ref); DRR is written as a copy of DDR."""
    D = _pts(D)
    ddr = np.zeros(bins ** 3, np.float64)
    rrr = np.zeros(bins ** 3, np.float64)
    ff = np.zeros(bins, np.float64)
    ffr = np.zeros(bins * bn_ref, np.float64)
    rc = lib().orc_analytic_3iso(_p(D), len(D), box, bins, dmax, ptt, bn_ref, int(wrap),
                                 _d(ddr), _d(rrr), _d(ff), _d(ffr))
    assert rc == 0
    s = (bins, bins, bins)
    return ddr.reshape(s), rrr.reshape(s), ff, ffr


def analytic_ff(D, *, box: float, bins: int, dmax: float, ptt: int = 100, bn_ref: int = 200,
                wrap: bool = True):
    """(ff_av, ff_av_ref, alpha_ref) of the analytic 3iso path, without the
    sub-grid refinement (use analytic_bin for single coarse bins)."""
    D = _pts(D)
    ff = np.zeros(bins, np.float64)
    ffr = np.zeros(bins * bn_ref, np.float64)
    a = np.zeros(1, np.float64)
    rc = lib().orc_analytic_ff(_p(D), len(D), box, bins, dmax, ptt, bn_ref, int(wrap), _d(ff),
                               _d(ffr), _d(a))
    assert rc == 0
    return ff, ffr, float(a[0])


def ff_average_ref(dd_ref, rr_ref, *, bins, dmax, ptt=100, bn_ref=200):
    """make_ff_av_ref of the analytic 3iso path (3isoBPC_k.cuh:2001) on given
    fine DD and RR histograms (ptt * bn_ref * bins bins): bn_ref * bins
    averaged correction factors."""
    dd = np.ascontiguousarray(dd_ref, np.float64)
    rr = np.ascontiguousarray(rr_ref, np.float64)
    assert dd.size == rr.size == ptt * bn_ref * bins
    out = np.zeros(bn_ref * bins, np.float64)
    lib().orc_ff_average_ref(_d(dd), _d(rr), bins, dmax, ptt, bn_ref, _d(out))
    return out


def analytic_bin(i, j, k, *, bins, dmax, bn_ref, alpha_ref, ff_ref):
    ffr = np.ascontiguousarray(ff_ref, np.float64)
    r = ctypes.c_double()
    d = ctypes.c_double()
    v = lib().orc_analytic_bin(i, j, k, bins, dmax, bn_ref, alpha_ref, _d(ffr),
                               ctypes.byref(r), ctypes.byref(d))
    return v, r.value, d.value


class RefEngine:
    """The reference's CPU NODE2P engine for one variant, compiled in place.

    kind: '2iso', '2iso_bpc', '2ani', '2ani_bpc'.
    """

    def __init__(self, kind: str):
        path = os.path.join(HERE, "_ref", f"libref_{kind}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.kind = kind
        self.lib = ctypes.CDLL(path)
        self.lib.ref_xx.argtypes = [_fptr, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                    ctypes.c_float, ctypes.c_int, _dptr]
        self.lib.ref_xy.argtypes = [_fptr, _fptr, ctypes.c_int, ctypes.c_float,
                                    ctypes.c_float, ctypes.c_float, ctypes.c_int, _dptr]
        self.is2d = bool(self.lib.ref_is_2d())

    def set_threads(self, t: int) -> None:
        self.lib.ref_set_threads(int(t))

    def xx(self, A, *, box, size_node, bins, dmax):
        A = _pts(A)
        out = np.zeros(bins * bins if self.is2d else bins, np.float64)
        self.lib.ref_xx(_p(A), len(A), box, size_node, dmax, bins, _d(out))
        return out.reshape(bins, bins) if self.is2d else out

    def xy(self, A, B, *, box, size_node, bins, dmax):
        A, B = _pts(A), _pts(B)
        assert len(A) == len(B), "the reference engines take catalogs of equal size"
        out = np.zeros(bins * bins if self.is2d else bins, np.float64)
        self.lib.ref_xy(_p(A), _p(B), len(A), box, size_node, dmax, bins, _d(out))
        return out.reshape(bins, bins) if self.is2d else out


def ref_read_catalog(path: str, n: int, box: float = 0.0):
    """The reference's own reader (open_files, cuda/create_grid.cuh:35-78,
    through _ref/libref_io.so) on the first n rows of `path`: (points as an
    (n, 4) float32 array, box).  box <= 0 asks for the reader's automatic box
    ceil(max component + 1).  The reader opens "../data/<name>" from the
    working directory, so the call runs from a scratch directory that links
    the file there."""
    import tempfile
    lib = ctypes.CDLL(os.path.join(HERE, "_ref", "libref_io.so"))
    lib.ref_open_files.argtypes = [ctypes.c_char_p, ctypes.c_int, _fptr,
                                   ctypes.POINTER(ctypes.c_float)]
    out = np.zeros((n, 4), np.float32)
    b = ctypes.c_float(box)
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as wd:
        os.makedirs(os.path.join(wd, "data"))
        os.makedirs(os.path.join(wd, "run"))
        os.symlink(os.path.abspath(path), os.path.join(wd, "data", "cat.dat"))
        os.chdir(os.path.join(wd, "run"))
        try:
            lib.ref_open_files(b"cat.dat", int(n), _p(out), ctypes.byref(b))
        finally:
            os.chdir(cwd)
    return out, float(b.value)


def ref_save_histogram(h, out_path: str) -> None:
    """Writes histogram h (bn, bn x bn or bn^3 doubles; dims from h.ndim)
    through the reference's own writers (save_histogram1D/2D/3D,
    cuda/create_grid.cuh:141-229, through _ref/libref_io.so) to out_path."""
    import shutil
    import tempfile
    lib = ctypes.CDLL(os.path.join(HERE, "_ref", "libref_io.so"))
    lib.ref_save_histogram.argtypes = [ctypes.c_int, ctypes.c_char_p, ctypes.c_int, _dptr]
    a = np.ascontiguousarray(h, dtype=np.float64)
    cwd = os.getcwd()
    with tempfile.TemporaryDirectory() as wd:
        os.makedirs(os.path.join(wd, "results"))
        os.makedirs(os.path.join(wd, "run"))
        os.chdir(os.path.join(wd, "run"))
        try:
            rc = lib.ref_save_histogram(a.ndim, b"h.dat", a.shape[0], _d(a))
        finally:
            os.chdir(cwd)
        if rc != 0:
            raise ValueError("1, 2 or 3 dimensions")
        shutil.copy(os.path.join(wd, "results", "h.dat"), out_path)


class RefAnalyticRR:
    """The reference's CPU periodic 2-point engine with the analytic RR
    (cpp/2PCFisotropic/BPC_analitic/2PCF.h), compiled in place."""

    def __init__(self):
        path = os.path.join(HERE, "_ref", "libref_2iso_analytic.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        self.lib.ref_dd_rr_analytic.argtypes = [_fptr, ctypes.c_int, ctypes.c_float,
                                                ctypes.c_float, ctypes.c_float, ctypes.c_int,
                                                _dptr, _dptr]

    def set_threads(self, t: int) -> None:
        self.lib.ref_set_threads(int(t))

    def dd_rr(self, A, *, box, size_node, bins, dmax):
        A = _pts(A)
        dd = np.zeros(bins, np.float64)
        rr = np.zeros(bins, np.float64)
        self.lib.ref_dd_rr_analytic(_p(A), len(A), box, size_node, dmax, bins, _d(dd), _d(rr))
        return dd, rr


class Ref3IsoBPC:
    """The reference's CPU periodic 3-point engine NODE3P
    (cpp/3PCFisotropic/BPC/3PCFiso.h), compiled in place: DDD of one
    catalog and the analytic path's averaged correction factors."""

    def __init__(self):
        path = os.path.join(HERE, "_ref", "libref_3iso_bpc.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        self.lib.ref3_xxx.argtypes = [_fptr, ctypes.c_int, ctypes.c_float, ctypes.c_float,
                                      ctypes.c_float, ctypes.c_int, _dptr]
        self.lib.ref3_analytic_ff.argtypes = [_fptr, ctypes.c_int, ctypes.c_float,
                                              ctypes.c_float, ctypes.c_float, ctypes.c_int,
                                              ctypes.c_char_p, _dptr, _dptr, _dptr]

    def set_threads(self, t: int) -> None:
        self.lib.ref_set_threads(int(t))

    def xxx(self, A, *, box, size_node, bins, dmax):
        A = _pts(A)
        out = np.zeros(bins ** 3, np.float64)
        self.lib.ref3_xxx(_p(A), len(A), box, size_node, dmax, bins, _d(out))
        return out.reshape(bins, bins, bins)

    def analytic_ff(self, A, *, box, size_node, bins, dmax, workdir):
        """(ff_av, ff_av_ref, fine DD of ff_av_ref at 100*200*bins bins); the
        engine writes them as text files into workdir."""
        A = _pts(A)
        ff = np.zeros(bins, np.float64)
        ffr = np.zeros(200 * bins, np.float64)
        dd = np.zeros(100 * 200 * bins, np.float64)
        rc = self.lib.ref3_analytic_ff(_p(A), len(A), box, size_node, dmax, bins,
                                       os.fsencode(workdir), _d(ff), _d(ffr), _d(dd))
        assert rc == 0
        return ff, ffr, dd


def available_ref_engines():
    d = os.path.join(HERE, "_ref")
    if not os.path.isdir(d):
        return []
    return sorted(f[len("libref_"):-3] for f in os.listdir(d) if f.startswith("libref_"))

def _kernels_lib():
    lib = ctypes.CDLL(os.path.join(HERE, "_ref", "libref_kernels_host.so"))
    args = [ctypes.c_int, ctypes.c_int, _fptr, ctypes.c_int, _fptr, ctypes.c_int, ctypes.c_int,
            ctypes.c_float, ctypes.c_int, ctypes.c_float, _dptr]
    lib.ref2_hist.argtypes = args
    lib.ref3_hist.argtypes = args
    return lib


def ref_kernels_available() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libref_kernels_host.so"))


def ref_kernels_3pt(D, R=None, *, ani: bool, bpc: bool, box: float, bins: int, dmax: float,
                    partitions: int):
    """The reference's own 3-point CUDA kernels (XXX3iso/XXY3iso,
    XXX3iso_BPC/XXY3iso_BPC, XXX3ani/XXY3ani, XXX3ani_BPC/XXY3ani_BPC in
    cuda/kernels/3{iso,ani}{,BPC}_k.cuh) compiled for the host
    (_ref/libref_kernels_host.so, ref_kernels_host.cpp), on nodes of
    box/partitions: {"DDD": ...} or, with R, {"DDD", "RRR", "DDR", "DRR"},
    each bins^3 (iso) or bins^5 (ani).  Unit weights only (see
    ref_kernels_host.cpp)."""
    D = _pts(D)
    Rp = _pts(R) if R is not None else None
    shape = (bins,) * (5 if ani else 3)
    nb = int(np.prod(shape))
    out = np.zeros(nb * (4 if Rp is not None else 1), np.float64)
    rc = _kernels_lib().ref3_hist(int(ani), int(bpc), _p(D), len(D), _p(Rp) if Rp is not None else None,
                                  len(Rp) if Rp is not None else 0, bins, dmax, partitions, box, _d(out))
    if rc != 0:
        raise ValueError(f"ref3_hist returned {rc} (a coordinate outside the node grid?)")
    names = ("DDD", "RRR", "DDR", "DRR") if Rp is not None else ("DDD",)
    return {k: out[i * nb:(i + 1) * nb].reshape(shape) for i, k in enumerate(names)}


def ref_kernels_2pt(D, R, *, ani: bool, bpc: bool, box: float, bins: int, dmax: float,
                    partitions: int):
    """The reference's own pair CUDA kernels (XX2iso/XY2iso,
    XX2iso_BPC/XY2iso_BPC, XX2ani, XX2ani_BPC in
    cuda/kernels/2{iso,ani}{,BPC}_k.cuh) compiled for the host, on nodes of
    box/partitions: {"DD", "RR", "DR"}, each bins (iso) or bins x bins (ani).
    The anisotropic DR is NaN: its kernels read an out-of-range weight
    (XY2ani) or an unset one (XY2ani_BPC), see ref_kernels_host.cpp."""
    D, Rp = _pts(D), _pts(R)
    shape = (bins, bins) if ani else (bins,)
    nb = int(np.prod(shape))
    out = np.zeros(3 * nb, np.float64)
    rc = _kernels_lib().ref2_hist(int(ani), int(bpc), _p(D), len(D), _p(Rp), len(Rp), bins, dmax,
                                  partitions, box, _d(out))
    if rc != 0:
        raise ValueError(f"ref2_hist returned {rc} (a coordinate outside the node grid?)")
    return {k: out[i * nb:(i + 1) * nb].reshape(shape) for i, k in enumerate(("DD", "RR", "DR"))}
