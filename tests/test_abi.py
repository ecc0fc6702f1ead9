"""CPU: the C-ABI library loads and exports every symbol include/pcf.h declares."""
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared(header):
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    names = re.findall(r"\b(pcf_[a-z0-9_]+)\s*\(", src)
    return sorted(set(n for n in names if not n.startswith("pcf_status")))


def test_library_exports_every_declared_symbol():
    from desi_b200 import _lib
    lib = _lib.lib()
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True).stdout
    headers = sorted(f for f in os.listdir(os.path.join(ROOT, "include")) if f.endswith(".h"))
    for h in headers:
        if h == "pcf_legacy.h":
            continue  # C++ signatures (mangled), checked by the legacy test
        missing = [n for n in _declared(h) if not hasattr(lib, n)]
        assert not missing, (h, missing)
        for n in _declared(h):
            assert re.search(rf"\bT {n}\b", out), n


def test_version_and_status_strings():
    from desi_b200 import _lib
    lib = _lib.lib()
    assert lib.pcf_version() >= 1
    assert lib.pcf_status_string(0) == b"ok"
    assert b"argument" in lib.pcf_status_string(-1)


def test_ctx_create_fails_cleanly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    import ctypes
    from desi_b200 import _lib
    h = ctypes.c_void_p()
    assert _lib.lib().pcf_ctx_create(0, ctypes.byref(h)) != 0


def test_alloc_counters_read_on_the_host():
    """pcf_alloc_counters (include/pcf_bench.h) reads process-wide counters
    without touching a device: six values, never decreasing."""
    from desi_b200 import _lib
    a = _lib.alloc_counters()
    assert set(a) == {"device_allocs", "device_bytes", "device_s", "host_allocs", "host_bytes",
                      "host_s"}
    assert all(v >= 0 for v in a.values())
    b = _lib.alloc_counters()
    assert all(b[k] >= a[k] for k in a)
    assert _lib.lib().pcf_alloc_counters(None) == -1  # PCF_ERR_INVALID_ARG
