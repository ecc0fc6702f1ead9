"""GPU: the no-allocation pair entry point (include/pcf_noalloc.h).

pcf_count_pairs_noalloc is for callers that cannot call cudaMalloc (for
example a plug-in host that owns the device memory budget, or code inside a
stream capture it does not control): all its scratch sits in one fixed array
of the library's device image.  Here it is called through the C ABI on
device-resident catalogs and must reproduce pcf_count_pairs -- bit for bit
with unit weights, within 1e-12 relative with weights (FP64 sums in another
order) -- on two calls in a row, since every call reuses the same array.
Collected last (file name) so a failure here cannot hide the other tests.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PCF_ERR_UNSUPPORTED = -4


def _noalloc(lib, torch, A, B, box, kind, bins, dmax, flags):
    nb = bins * bins if kind == 1 else bins
    out = torch.zeros(nb, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    rc = lib.pcf_count_pairs_noalloc(
        ctypes.c_void_p(A.data_ptr()), A.shape[0],
        ctypes.c_void_p(B.data_ptr()) if B is not None else None, B.shape[0] if B is not None else 0,
        box, kind, bins, dmax, flags, ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))
    torch.cuda.synchronize()
    return rc, out.cpu().numpy()


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
                        if weights == "unit":
                            assert np.array_equal(got, want)
                        else:
                            np.testing.assert_allclose(got, want, rtol=1e-12, atol=0)
    finally:
        ctx.close()


def test_no_alloc_rejects_inputs_beyond_its_scratch():
    import torch

    from desi_b200 import _lib, catalog

    lib = _lib.lib()
    big = torch.from_numpy(catalog.uniform(400_000, 250.0, seed=43)).cuda()
    rc, _ = _noalloc(lib, torch, big, None, 250.0, 0, 30, 80.0, 0)
    assert rc == PCF_ERR_UNSUPPORTED
