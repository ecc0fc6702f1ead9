"""GPU: the entry point that allocates nothing (include/pcf_noalloc.h).

pcf_count_pairs_noalloc is for callers that may not allocate device memory:
plug-in hosts that own the device memory budget and forbid the libraries
they load from calling cudaMalloc, and processes whose allocator is at its
limit, where a per-call allocation would fail midway.  All its scratch sits
in one fixed array in the library's device image.  Here it is called
through the C ABI on device-resident catalogs and must reproduce the
existing entry point pcf_count_pairs -- bit for bit with unit weights,
within 1e-12 relative with weights (FP64 sums in another order) -- on two
calls in a row, since every call reuses the same array; one case is also
checked against the FP64 oracle, and the device's free memory must not move
across the calls.  The file name makes pytest collect it last, so a failure
here cannot hide the other tests.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PCF_ERR_UNSUPPORTED = -4


def _noalloc(lib, torch, A, B, box, kind, bins, dmax, flags, out=None):
    nb = bins * bins if kind == 1 else bins
    if out is None:
        out = torch.zeros(nb, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.pcf_count_pairs_noalloc(
        ctypes.c_void_p(A.data_ptr()), A.shape[0],
        ctypes.c_void_p(B.data_ptr()) if B is not None else None, B.shape[0] if B is not None else 0,
        box, kind, bins, dmax, flags, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
    torch.cuda.synchronize()
    return rc, out


@pytest.mark.parametrize("weights", ["unit", "uniform"])
def test_no_alloc_matches_pcf_count_pairs(weights):
    import torch

    from desi_b200 import _lib, api, catalog

    lib = _lib.lib()
    box, bins, dmax = 250.0, 30, 80.0
    D = catalog.neyman_scott(6000, box, seed=41, weights=weights)
    R = catalog.uniform(7000, box, seed=42, weights=weights)
    Dt = torch.from_numpy(D).cuda()
    Rt = torch.from_numpy(R).cuda()
    ctx = api.Context(0)
    try:
        gd, gr = ctx.grid(D, box), ctx.grid(R, box)
        for kind in (0, 1):
            for bpc in (False, True):
                flags = api.PCF_BPC if bpc else 0
                for (A, B, ga, gb) in ((Dt, None, gd, None), (Dt, Rt, gd, gr)):
                    want = ctx.count_pairs(ga, gb, bins=bins, dmax=dmax, ani=kind == 1, bpc=bpc)
                    want = np.asarray(want).reshape(-1)
                    for _ in range(2):  # the shared scratch keeps the last call's contents
                        rc, got = _noalloc(lib, torch, A, B, box, kind, bins, dmax, flags)
                        assert rc == 0
                        got = got.cpu().numpy()
                        if weights == "unit":
                            assert np.array_equal(got, want)
                        else:
                            np.testing.assert_allclose(got, want, rtol=1e-12, atol=0)
    finally:
        ctx.close()


def test_no_alloc_matches_oracle_and_leaves_device_memory_alone():
    """Periodic weighted DR against the FP64 oracle (1e-12), and the
    device's free memory and the caching allocator's reserve unchanged by
    two further calls (output buffer allocated beforehand)."""
    import torch

    import oracle
    from desi_b200 import _lib, catalog

    lib = _lib.lib()
    box, bins, dmax = 250.0, 30, 80.0
    D = catalog.neyman_scott(5000, box, seed=51, weights="uniform")
    R = catalog.uniform(5500, box, seed=52, weights="uniform")
    Dt, Rt = torch.from_numpy(D).cuda(), torch.from_numpy(R).cuda()
    out = torch.zeros(bins, dtype=torch.float64, device="cuda")
    rc, _ = _noalloc(lib, torch, Dt, Rt, box, 0, bins, dmax, 1, out)  # first call: set-up
    assert rc == 0
    free0, _ = torch.cuda.mem_get_info()
    res0 = torch.cuda.memory_reserved()
    for _ in range(2):
        rc, _ = _noalloc(lib, torch, Dt, Rt, box, 0, bins, dmax, 1, out)
        assert rc == 0
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.cuda.memory_reserved() == res0
    want = oracle.pairs(D, R, box=box, bins=bins, dmax=dmax, bpc=True)
    np.testing.assert_allclose(out.cpu().numpy(), want, rtol=1e-12, atol=0)


def test_no_alloc_rejects_inputs_beyond_its_scratch():
    import torch

    from desi_b200 import _lib, catalog

    lib = _lib.lib()
    big = torch.from_numpy(catalog.uniform(400_000, 250.0, seed=43)).cuda()
    rc, _ = _noalloc(lib, torch, big, None, 250.0, 0, 30, 80.0, 0)
    assert rc == PCF_ERR_UNSUPPORTED
    # an anisotropic histogram of more than 2^24 bins (5000^2) is refused
    # before any scratch is carved
    small = torch.from_numpy(catalog.uniform(1000, 250.0, seed=44)).cuda()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    rc, _ = _noalloc(lib, torch, small, None, 250.0, 1, 5000, 80.0, 0, out)
    assert rc == PCF_ERR_UNSUPPORTED
