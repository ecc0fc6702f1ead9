"""Python view of libpcf (tests, bench and scripting).

Thin wrappers over the C ABI of ``include/pcf.h``: a :class:`Context` owns a
CUDA stream; :class:`Grid` is a catalog gridded on the device; the
``count_*`` functions return numpy histograms laid out exactly like the
reference's (``[bin]``, ``[bin_z][bin_perp]``, ``[b12][b23][b31]``).
Every call goes to the CUDA library; errors raise :class:`PcfError`.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from ._lib import (PCF_ANI, PCF_BOTH, PCF_BPC, PCF_DEVICE_OUT, PCF_DS_EXACT,  # noqa: F401
                   PCF_ERR_TIMEOUT, PCF_GRAPH, PCF_ISO, PCF_OPT_ABORT_HOST_CHECK,
                   PCF_OPT_GRID_BUILD, PCF_OPT_GRID_DEFER, PCF_OPT_PAIR_VARIANT,
                   PCF_OPT_TRIP_FLUSH_BUDGET, PCF_REF_NODE_GATES,
                   PCF_RULE_CUSTOM, PCF_RULE_EXCL_ZERO, PCF_RULE_INCLUSIVE, PcfError, Stats)


def _check(ctx, rc, where):
    if rc != 0:
        detail = ""
        if ctx is not None:
            try:
                detail = (_lib.lib().pcf_last_error(ctx) or b"").decode()
            except Exception:  # pragma: no cover
                detail = ""
        raise PcfError(rc, where, detail)


def as_points(a) -> np.ndarray:
    """(n, 4) float32 C-contiguous array (x, y, z, w)."""
    a = np.ascontiguousarray(a, dtype=np.float32)
    if a.ndim != 2 or a.shape[1] not in (3, 4):
        raise ValueError("points must be (n, 4) [x, y, z, w] or (n, 3)")
    if a.shape[1] == 3:
        a = np.ascontiguousarray(np.concatenate([a, np.ones((len(a), 1), np.float32)], axis=1))
    return a


class Context:
    """One CUDA stream on one device; owns the grids it builds."""

    def __init__(self, device: int = 0):
        self._lib = _lib.lib()
        h = ctypes.c_void_p()
        _check(None, self._lib.pcf_ctx_create(device, ctypes.byref(h)), "pcf_ctx_create")
        self.handle = h
        self.device = device

    @property
    def stream(self) -> int:
        return int(self._lib.pcf_ctx_stream(self.handle) or 0)

    # -- failure handling ------------------------------------------------------
    def abort(self, on: bool = True) -> None:
        """Ask this context's running and future kernels to stop taking work
        (calls then raise PcfError(PCF_ERR_TIMEOUT)); abort(False) clears the
        request.  Safe to call from another thread while a call runs."""
        _check(self.handle, self._lib.pcf_ctx_abort(self.handle, int(bool(on))), "pcf_ctx_abort")

    def synchronize(self) -> None:
        """Wait for the context stream; raises PcfError(PCF_ERR_TIMEOUT) if a
        kernel gave up its queue since the last abort(False)."""
        _check(self.handle, self._lib.pcf_ctx_synchronize(self.handle), "pcf_ctx_synchronize")

    def set_option(self, option: int, value: int) -> None:
        """pcf_ctx_set_option (include/pcf_bench.h): PCF_OPT_TRIP_FLUSH_BUDGET,
        PCF_OPT_ABORT_HOST_CHECK, PCF_OPT_PAIR_VARIANT, PCF_OPT_GRID_BUILD, PCF_OPT_GRID_DEFER."""
        _check(self.handle, self._lib.pcf_ctx_set_option(self.handle, int(option), int(value)),
               "pcf_ctx_set_option")

    def close(self):
        if self.handle:
            self._lib.pcf_ctx_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):  # pragma: no cover
        try:
            self.close()
        except Exception:
            pass

    # -- grids ---------------------------------------------------------------
    def grid(self, points, box: float, partitions: int = 0, device_ptr: int | None = None,
             n: int | None = None) -> "Grid":
        """Grid a catalog.  ``points``: (n,4) array on the host, or pass
        ``device_ptr``/``n`` for points already in device memory (a torch
        CUDA tensor's ``data_ptr()``)."""
        if device_ptr is not None:
            ptr, count, keep = ctypes.c_void_p(device_ptr), int(n), None
        else:
            keep = as_points(points)
            ptr, count = keep.ctypes.data_as(ctypes.c_void_p), len(keep)
        h = ctypes.c_void_p()
        _check(self.handle,
               self._lib.pcf_grid_build(self.handle, ptr, count, float(box), int(partitions),
                                        ctypes.byref(h)), "pcf_grid_build")
        g = Grid(self, h, count, float(box))
        g._points = keep  # a deferred build reads them until its first use
        return g

    # -- counting ------------------------------------------------------------
    def count_pairs(self, a: "Grid", b: "Grid | None" = None, *, bins: int, dmax: float,
                    ani: "bool | str" = False, bpc: bool = False, flags: int = 0,
                    stats: bool = False, out_device_ptr: int | None = None):
        """One pair histogram (DD / RR with b None, else DR).  ani=False:
        isotropic [bins]; True: anisotropic [bins, bins]; "both": the two in
        one call (one pass over the candidates where the autotuner found that
        faster), returned as (iso, ani) (a device output then holds bins +
        bins^2 doubles, isotropic first)."""
        both = ani == "both"
        kind = PCF_BOTH if both else (PCF_ANI if ani else PCF_ISO)
        nb = bins + bins * bins if both else (bins * bins if ani else bins)
        f = flags | (PCF_BPC if bpc else 0)
        st = Stats()
        if out_device_ptr is not None:
            f |= PCF_DEVICE_OUT
            outp = ctypes.c_void_p(out_device_ptr)
            out = None
        else:
            out = np.zeros(nb, np.float64)
            outp = out.ctypes.data_as(ctypes.c_void_p)
        rc = self._lib.pcf_count_pairs(self.handle, kind, a.handle,
                                       b.handle if b is not None else None, int(bins),
                                       float(dmax), f, outp, ctypes.byref(st) if stats else None)
        _check(self.handle, rc, "pcf_count_pairs")
        if out is not None and both:
            out = (out[:bins], out[bins:].reshape(bins, bins))
        elif out is not None and ani:
            out = out.reshape(bins, bins)
        return (out, st.as_dict()) if stats else out

    def count_triplets(self, x: "Grid", y: "Grid | None" = None, *, bins: int, dmax: float,
                       ani: bool = False, bpc: bool = False, flags: int = 0,
                       stats: bool = False, out_device_ptr: int | None = None,
                       ref_gates: bool = False):
        """One triplet histogram (XXX with y None, else XXY); out_device_ptr:
        write it to device memory without waiting for it (isotropic only).
        ref_gates (periodic): count as the reference's periodic CUDA kernels
        do on the node grid of the partitions the grids were built with
        (PCF_REF_NODE_GATES)."""
        nb = bins ** 5 if ani else bins ** 3
        st = Stats()
        f = flags | (PCF_BPC if bpc else 0) | (PCF_REF_NODE_GATES if ref_gates else 0)
        if out_device_ptr is not None:
            f |= PCF_DEVICE_OUT
            out, outp = None, ctypes.c_void_p(out_device_ptr)
        else:
            out = np.zeros(nb, np.float64)
            outp = out.ctypes.data_as(ctypes.c_void_p)
        rc = self._lib.pcf_count_triplets(self.handle, PCF_ANI if ani else PCF_ISO, x.handle,
                                          y.handle if y is not None else None, int(bins),
                                          float(dmax), f, outp,
                                          ctypes.byref(st) if stats else None)
        _check(self.handle, rc, "pcf_count_triplets")
        if out is not None:
            out = out.reshape((bins,) * (5 if ani else 3))
        return (out, st.as_dict()) if stats else out

    def analytic_rr(self, bins: int, n: int, box: float, dmax: float, wrap: bool = True):
        out = np.zeros(bins, np.float64)
        rc = self._lib.pcf_analytic_rr(self.handle, int(bins), int(n), float(box), float(dmax),
                                       int(wrap), out.ctypes.data_as(ctypes.c_void_p))
        _check(self.handle, rc, "pcf_analytic_rr")
        return out

    def analytic_3iso(self, d: "Grid", *, bins: int, dmax: float, ptt: int = 100,
                      bn_ref: int = 200, wrap: bool = True, with_ddd: bool = True,
                      stats: bool = False):
        n3 = bins ** 3
        ddd = np.zeros(n3, np.float64) if with_ddd else None
        ddr = np.zeros(n3, np.float64)
        rrr = np.zeros(n3, np.float64)
        st = Stats()
        rc = self._lib.pcf_analytic_3iso(
            self.handle, d.handle, int(bins), float(dmax), int(ptt), int(bn_ref), int(wrap),
            ddd.ctypes.data_as(ctypes.c_void_p) if ddd is not None else None,
            ddr.ctypes.data_as(ctypes.c_void_p), rrr.ctypes.data_as(ctypes.c_void_p),
            ctypes.byref(st))
        _check(self.handle, rc, "pcf_analytic_3iso")
        s = (bins, bins, bins)
        res = (ddd.reshape(s) if ddd is not None else None, ddr.reshape(s), rrr.reshape(s))
        return (res, st.as_dict()) if stats else res

    def batch_pairs(self, d: "Grid", rands, *, bins: int, dmax: float, ani: "bool | str" = False,
                    bpc: bool = False, flags: int = 0, want_dd: bool = True,
                    stats: bool = False, graph: bool = False):
        """DD, RR_i and DR_i of one data grid against random grids in one
        launch.  ani as for count_pairs ("both": each result an (iso, ani) pair)."""
        nr = len(rands)
        both = ani == "both"
        kind = PCF_BOTH if both else (PCF_ANI if ani else PCF_ISO)
        nb = bins + bins * bins if both else (bins * bins if ani else bins)
        arr = (ctypes.c_void_p * nr)(*[r.handle.value for r in rands])
        dd = np.zeros(nb, np.float64) if want_dd else None
        rr = np.zeros(nr * nb, np.float64)
        dr = np.zeros(nr * nb, np.float64)
        st = Stats()
        f = flags | (PCF_BPC if bpc else 0) | (PCF_GRAPH if graph else 0)
        rc = self._lib.pcf_batch_pairs(self.handle, kind, d.handle,
                                       ctypes.cast(arr, ctypes.c_void_p), nr, int(bins),
                                       float(dmax), f,
                                       dd.ctypes.data_as(ctypes.c_void_p) if dd is not None else None,
                                       rr.ctypes.data_as(ctypes.c_void_p),
                                       dr.ctypes.data_as(ctypes.c_void_p), ctypes.byref(st))
        _check(self.handle, rc, "pcf_batch_pairs")
        if both:
            rr, dr = rr.reshape(nr, nb), dr.reshape(nr, nb)
            split = lambda h: (h[..., :bins], h[..., bins:].reshape(h.shape[:-1] + (bins, bins)))
            res = (split(dd) if dd is not None else None, split(rr), split(dr))
            return (res, st.as_dict()) if stats else res
        shp = (nr, bins, bins) if ani else (nr, bins)
        if dd is not None and ani:
            dd = dd.reshape(bins, bins)
        res = (dd, rr.reshape(shp), dr.reshape(shp))
        return (res, st.as_dict()) if stats else res

    def batch_triplets(self, d: "Grid", rands, *, bins: int, dmax: float, bpc: bool = False,
                       flags: int = 0, stats: bool = False):
        """DDD, and RRR_i, DDR_i, DRR_i per random grid, in one persistent
        launch (pcf_batch_triplets): (ddd, rrr, ddr, drr), the last three
        with a leading random-catalog axis."""
        nr = len(rands)
        n3 = bins ** 3
        arr = (ctypes.c_void_p * max(nr, 1))(*[r.handle.value for r in rands])
        ddd = np.zeros(n3, np.float64)
        rrr, ddr, drr = (np.zeros(max(nr, 1) * n3, np.float64) for _ in range(3))
        st = Stats()
        f = flags | (PCF_BPC if bpc else 0)
        p = lambda x: x.ctypes.data_as(ctypes.c_void_p)  # noqa: E731
        rc = self._lib.pcf_batch_triplets(self.handle, d.handle, ctypes.cast(arr, ctypes.c_void_p),
                                          nr, int(bins), float(dmax), f, p(ddd), p(rrr), p(ddr),
                                          p(drr), ctypes.byref(st))
        _check(self.handle, rc, "pcf_batch_triplets")
        shp = (nr, bins, bins, bins)
        res = (ddd.reshape(bins, bins, bins), rrr[:nr * n3].reshape(shp), ddr[:nr * n3].reshape(shp),
               drr[:nr * n3].reshape(shp))
        return (res, st.as_dict()) if stats else res

    def estimate(self, hists, n_d: int = 0, n_r: int = 0) -> np.ndarray:
        """Landy-Szalay: hists = (DD, DR, RR) or (DDD, DDR, DRR, RRR)."""
        hs = [np.ascontiguousarray(h, np.float64) for h in hists]
        shape = hs[0].shape
        out = np.zeros(hs[0].size, np.float64)
        p = [h.ctypes.data_as(ctypes.c_void_p) for h in hs] + [None] * (4 - len(hs))
        npoint = 2 if len(hs) == 3 else 3
        _check(self.handle, self._lib.pcf_estimate(self.handle, npoint, hs[0].size, *p, int(n_d),
                                                   int(n_r), out.ctypes.data_as(ctypes.c_void_p)),
               "pcf_estimate")
        return out.reshape(shape)

    def autotune_pairs(self, a: "Grid", b: "Grid | None" = None, *, bins: int, dmax: float,
                       ani: bool = False, bpc: bool = False, flags: int = 0) -> dict:
        """Time launch shapes on these catalogs; later counts of the class use the winner."""
        r = _lib.TuneResult()
        f = flags | (PCF_BPC if bpc else 0)
        _check(self.handle, self._lib.pcf_autotune_pairs(
            self.handle, PCF_BOTH if ani == "both" else (PCF_ANI if ani else PCF_ISO), a.handle,
            b.handle if b is not None else None,
            int(bins), float(dmax), f, ctypes.byref(r)), "pcf_autotune_pairs")
        return r.as_dict()

    def tune_save(self, path: str) -> None:
        _check(self.handle, self._lib.pcf_tune_save(self.handle, path.encode()), "pcf_tune_save")

    def tune_load(self, path: str) -> None:
        _check(self.handle, self._lib.pcf_tune_load(self.handle, path.encode()), "pcf_tune_load")

    @property
    def tune_size(self) -> int:
        return int(self._lib.pcf_tune_size(self.handle))

    def microbench(self, which: int) -> float:
        """0: FP32 FMA TFLOP/s; 1: conflict-free shared atomic Gop/s."""
        r = ctypes.c_double()
        _check(self.handle, self._lib.pcf_microbench(self.handle, int(which), ctypes.byref(r)),
               "pcf_microbench")
        return r.value

    def profile(self, enable: bool = True) -> None:
        """Start (or stop) logging the device time of every counting kernel."""
        _check(self.handle, self._lib.pcf_ctx_profile(self.handle, int(enable)), "pcf_ctx_profile")

    def profile_read(self):
        """(summed kernel ms, logged launches) since profile(); clears the log."""
        ms = ctypes.c_double()
        n = ctypes.c_int64()
        _check(self.handle, self._lib.pcf_ctx_profile_read(self.handle, ctypes.byref(ms),
                                                           ctypes.byref(n)), "pcf_ctx_profile_read")
        return ms.value, n.value

    def profile_read_grid(self):
        """(summed grid-build kernel ms, builds, points gridded) since
        profile(); clears that log."""
        ms = ctypes.c_double()
        n = ctypes.c_int64()
        pts = ctypes.c_int64()
        _check(self.handle, self._lib.pcf_ctx_profile_read_grid(self.handle, ctypes.byref(ms),
                                                                ctypes.byref(n), ctypes.byref(pts)),
               "pcf_ctx_profile_read_grid")
        return ms.value, n.value, pts.value

    @property
    def launches(self) -> int:
        return int(self._lib.pcf_ctx_launch_count(self.handle))

    def autotune_partitions(self, n, box, dmax, ani=False, bpc=False):
        return self._lib.pcf_autotune_partitions(self.handle, int(n), float(box), float(dmax),
                                                 PCF_ANI if ani else PCF_ISO,
                                                 PCF_BPC if bpc else 0)


class Grid:
    def __init__(self, ctx: Context, handle, n: int, box: float):
        self.ctx = ctx
        self.handle = handle
        self.n = n
        self.box = box

    def info(self):
        n = ctypes.c_int64()
        box = ctypes.c_float()
        p = ctypes.c_int()
        ne = ctypes.c_int64()
        uw = ctypes.c_int()
        _check(self.ctx.handle, self.ctx._lib.pcf_grid_info(self.handle, ctypes.byref(n),
                                                            ctypes.byref(box), ctypes.byref(p),
                                                            ctypes.byref(ne), ctypes.byref(uw)),
               "pcf_grid_info")
        return {"n": n.value, "box": box.value, "partitions": p.value,
                "nonempty_cells": ne.value, "unit_weights": bool(uw.value)}

    def download(self):
        info = self.info()
        P = info["partitions"]
        pts = np.zeros((self.n, 4), np.float32)
        cs = np.zeros(P ** 3 + 1, np.int32)
        _check(self.ctx.handle,
               self.ctx._lib.pcf_grid_download(self.ctx.handle, self.handle,
                                               pts.ctypes.data_as(ctypes.c_void_p),
                                               cs.ctypes.data_as(ctypes.c_void_p)),
               "pcf_grid_download")
        return pts, cs

    def free(self):
        if self.handle:
            self.ctx._lib.pcf_grid_free(self.ctx.handle, self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover
        try:
            if self.handle and self.ctx.handle:
                self.free()
        except Exception:
            pass
