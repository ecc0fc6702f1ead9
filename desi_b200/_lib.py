"""ctypes binding of libpcf.so (include/pcf.h).

The CUDA library is the only compute path: if ``libpcf.so`` is missing or
fails to load, importing this module raises -- there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libpcf.so")

PCF_ISO, PCF_ANI, PCF_BOTH = 0, 1, 2
PCF_BPC = 1 << 0
PCF_DS_EXACT = 1 << 1
PCF_RULE_CUSTOM = 1 << 2
PCF_RULE_EXCL_ZERO = 1 << 3
PCF_RULE_INCLUSIVE = 1 << 4
PCF_DEVICE_OUT = 1 << 5
PCF_GRAPH = 1 << 7
PCF_REF_NODE_GATES = 1 << 8
PCF_ERR_TIMEOUT = -6
(PCF_OPT_TRIP_FLUSH_BUDGET, PCF_OPT_ABORT_HOST_CHECK, PCF_OPT_PAIR_VARIANT, PCF_OPT_GRID_BUILD,
 PCF_OPT_GRID_DEFER) = 1, 2, 3, 4, 5

STATUS = {0: "ok", -1: "invalid argument", -2: "CUDA error", -3: "out of memory",
          -4: "unsupported configuration", -5: "coordinate outside [0, box)",
          -6: "device wait timed out", -7: "I/O error", -8: "grids do not match"}


class PcfError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        msg = f"{where}: {STATUS.get(status, status)}"
        if detail:
            msg += f" ({detail})"
        super().__init__(msg)


class TuneResult(ctypes.Structure):
    _fields_ = [("refine", ctypes.c_int), ("hist_mode", ctypes.c_int), ("best_ms", ctypes.c_float),
                ("default_ms", ctypes.c_float), ("tried", ctypes.c_int), ("tile", ctypes.c_int),
                ("chunk", ctypes.c_int)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class Stats(ctypes.Structure):
    _fields_ = [("pairs", ctypes.c_double), ("candidates", ctypes.c_double),
                ("rechecks", ctypes.c_double), ("kernel_ms", ctypes.c_float),
                ("partitions", ctypes.c_int), ("work_items", ctypes.c_int)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_vp = ctypes.c_void_p
_dp = ctypes.POINTER(ctypes.c_double)
_i64 = ctypes.c_int64

# name -> (restype, argtypes)
_SIGS = {
    "pcf_version": (ctypes.c_int, []),
    "pcf_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "pcf_last_error": (ctypes.c_char_p, [_vp]),
    "pcf_ctx_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_vp)]),
    "pcf_ctx_destroy": (ctypes.c_int, [_vp]),
    "pcf_ctx_stream": (_vp, [_vp]),
    "pcf_grid_build": (ctypes.c_int, [_vp, _vp, _i64, ctypes.c_float, ctypes.c_int,
                                      ctypes.POINTER(_vp)]),
    "pcf_grid_free": (ctypes.c_int, [_vp, _vp]),
    "pcf_grid_info": (ctypes.c_int, [_vp, ctypes.POINTER(_i64), ctypes.POINTER(ctypes.c_float),
                                     ctypes.POINTER(ctypes.c_int), ctypes.POINTER(_i64),
                                     ctypes.POINTER(ctypes.c_int)]),
    "pcf_grid_download": (ctypes.c_int, [_vp, _vp, _vp, _vp]),
    "pcf_count_pairs": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.c_int, ctypes.c_float,
                                       ctypes.c_uint32, _vp, ctypes.POINTER(Stats)]),
    "pcf_count_triplets": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.c_int,
                                          ctypes.c_float, ctypes.c_uint32, _vp,
                                          ctypes.POINTER(Stats)]),
    "pcf_analytic_rr": (ctypes.c_int, [_vp, ctypes.c_int, _i64, ctypes.c_float, ctypes.c_float,
                                       ctypes.c_int, _vp]),
    "pcf_analytic_3iso": (ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_float, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, _vp, _vp, _vp,
                                         ctypes.POINTER(Stats)]),
    "pcf_batch_pairs": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_float, ctypes.c_uint32, _vp, _vp, _vp,
                                       ctypes.POINTER(Stats)]),
    "pcf_batch_triplets": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                          ctypes.c_uint32, _vp, _vp, _vp, _vp,
                                          ctypes.POINTER(Stats)]),
    "pcf_autotune_partitions": (ctypes.c_int, [_vp, _i64, ctypes.c_float, ctypes.c_float,
                                               ctypes.c_int, ctypes.c_uint32]),
    "pcf_microbench": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.POINTER(ctypes.c_double)]),
    "pcf_count_pairs_noalloc": (ctypes.c_int, [_vp, _i64, _vp, _i64, ctypes.c_float, ctypes.c_int,
                                               ctypes.c_int, ctypes.c_float, ctypes.c_uint32, _vp,
                                               _vp]),
    "pcf_ctx_launch_count": (_i64, [_vp]),
    "pcf_read_catalog": (ctypes.c_int, [ctypes.c_char_p, _i64, _vp, ctypes.POINTER(_i64),
                                        ctypes.POINTER(ctypes.c_float)]),
    "pcf_write_catalog_f4": (ctypes.c_int, [ctypes.c_char_p, _vp, _i64]),
    "pcf_autotune_pairs": (ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp, ctypes.c_int, ctypes.c_float,
                                          ctypes.c_uint32, _vp]),
    "pcf_tune_save": (ctypes.c_int, [_vp, ctypes.c_char_p]),
    "pcf_tune_load": (ctypes.c_int, [_vp, ctypes.c_char_p]),
    "pcf_tune_size": (ctypes.c_int, [_vp]),
    "pcf_estimate": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _vp, _vp, _vp, _vp, _i64, _i64,
                                    _vp]),
    "pcf_ctx_abort": (ctypes.c_int, [_vp, ctypes.c_int]),
    "pcf_ctx_synchronize": (ctypes.c_int, [_vp]),
    "pcf_ctx_set_option": (ctypes.c_int, [_vp, ctypes.c_int, _i64]),
    "pcf_ctx_profile": (ctypes.c_int, [_vp, ctypes.c_int]),
    "pcf_ctx_profile_read": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_double),
                                            ctypes.POINTER(_i64)]),
    "pcf_ctx_profile_read_grid": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_double),
                                                 ctypes.POINTER(_i64), ctypes.POINTER(_i64)]),
    "pcf_alloc_counters": (ctypes.c_int, [ctypes.POINTER(ctypes.c_uint64)]),
}


def alloc_counters() -> dict:
    """Process-wide allocation counters of the library (pcf_alloc_counters):
    device and page-locked host allocations, their bytes and the seconds
    spent in those calls."""
    out = (ctypes.c_uint64 * 6)()
    lib().pcf_alloc_counters(out)
    return {"device_allocs": out[0], "device_bytes": out[1], "device_s": out[2] * 1e-9,
            "host_allocs": out[3], "host_bytes": out[4], "host_s": out[5] * 1e-9}


def exported_symbols():
    return list(_SIGS)


def load(path: str = LIB_PATH) -> ctypes.CDLL:
    if not os.path.exists(path):
        raise ImportError(f"libpcf.so not built at {path}: run python -m desi_b200.build")
    lib = ctypes.CDLL(path)
    for name, (res, args) in _SIGS.items():
        fn = getattr(lib, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    return lib


_lib = None


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        _lib = load()
    return _lib
