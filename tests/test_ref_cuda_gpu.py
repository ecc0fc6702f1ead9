"""The reference's own CUDA program (oracle/_ref/PCF_ref_cuda.out, built
unmodified from cuda/main.cu by oracle/Makefile) against this library's
PCF.out on the same files and flags: `3iso -bpc` and `3ani -bpc`, clustered
and uniform float catalogs, unit weights.  Periodic triplets count through
the reference kernels' node gates by default (PCF_REF_NODE_GATES), so the
histograms are the reference's bin for bin; -exact counts every triangle in
range once, which is more."""
import os
import tempfile

import numpy as np
import pytest

from desi_b200 import catalog
from oracle import ref_cuda

pytestmark = pytest.mark.gpu
OURS = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "desi_b200", "PCF.out")


def _cats(n, box):
    D = ref_cuda.inside_box(catalog.neyman_scott(n, box, seed=11), box)
    R = ref_cuda.inside_box(catalog.uniform(n, box, seed=12), box)
    D[:, 3] = 1.0
    R[:, 3] = 1.0
    return D, R


@pytest.mark.parametrize("kind,bins,dmax", [("3iso", 20, 60.0), ("3ani", 6, 40.0)])
def test_pcf_out_equals_reference_program(kind, bins, dmax):
    if not ref_cuda.available():
        pytest.skip("oracle/_ref/PCF_ref_cuda.out not built")
    box, n, P = 250.0, 2048, 20
    D, R = _cats(n, box)
    runs = {}
    for who, exe, extra in (("ref", None, ()), ("ours", OURS, ()), ("exact", OURS, ("-exact",))):
        with tempfile.TemporaryDirectory() as wd:
            runs[who] = ref_cuda.run_3pt_bpc(kind, D, R, box, bins, dmax, P, wd, exe=exe, extra=extra,
                                             timeout=300)
    for h in ("DDD", "RRR", "DDR", "DRR"):
        ref = runs["ref"][h]
        assert ref.sum() > 0, h
        # the reference's 3ani writer keeps the first bins^3 of bins^5 values
        assert np.array_equal(runs["ours"][h][:ref.size], ref), h
        assert runs["exact"][h][:ref.size].sum() >= ref.sum(), h
    if kind == "3iso":
        assert runs["exact"]["DDD"].sum() > runs["ref"]["DDD"].sum()
