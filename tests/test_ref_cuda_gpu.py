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


@pytest.mark.parametrize("kind", ["2iso", "2ani"])
def test_pcf_out_pairs_equal_reference_program(kind):
    """`2iso -bpc` and `2ani -bpc` of the reference's program and of this
    PCF.out on lattice catalogs (integer coordinates of a 60 box, weights in
    {0.5, 1, 1.5, 2}: every FP32 separation and weight product, and every
    sum, is exact in both) are equal bit for bit: DD, RR and DR, and for 2ani
    DD and RR (the reference's XY2ani_BPC weights most pairs by an unset
    variable, 2aniBPC_k.cuh:410)."""
    if not ref_cuda.available():
        pytest.skip("oracle/_ref/PCF_ref_cuda.out not built")
    rng = np.random.default_rng(77)
    n, box, bins, dmax, P = 3000, 60.0, 10, 20.0, 12
    D = np.empty((n, 4), np.float32)
    R = np.empty((n, 4), np.float32)
    D[:, :3] = 2 * rng.integers(0, 30, size=(n, 3))
    R[:, :3] = 2 * rng.integers(0, 30, size=(n, 3)) + 1
    D[:, 3] = rng.choice([0.5, 1.0, 1.5, 2.0], n)
    R[:, 3] = rng.choice([0.5, 1.0, 1.5, 2.0], n)
    runs = {}
    for who, exe in (("ref", None), ("ours", OURS)):
        with tempfile.TemporaryDirectory() as wd:
            runs[who] = ref_cuda.run_2pt_bpc(kind, D, R, box, bins, dmax, P, wd, exe=exe, timeout=300)
    for h in ("DD", "RR") + (("DR",) if kind == "2iso" else ()):
        assert runs["ref"][h].sum() > 0, h
        assert np.array_equal(runs["ours"][h], runs["ref"][h]), h


def _lattice(n, seed, weights):
    rng = np.random.default_rng(seed)
    D = np.empty((n, 4), np.float32)
    R = np.empty((n, 4), np.float32)
    D[:, :3] = 2 * rng.integers(0, 30, size=(n, 3))
    R[:, :3] = 2 * rng.integers(0, 30, size=(n, 3)) + 1
    D[:, 3] = rng.choice(weights, n)
    R[:, 3] = rng.choice(weights, n)
    return D, R


@pytest.mark.parametrize("kind", ["2iso", "2ani", "3iso", "3ani"])
def test_pcf_out_plain_equals_reference_program(kind):
    """The plain paths (no -bpc) of the reference's program and of this
    PCF.out on lattice catalogs of a 60 box, where every FP32 separation is
    exact: every histogram equal bit for bit.  Weights in {0.5, 1, 1.5, 2}
    for 2iso; unit weights for 2ani (the reference's XY2ani takes the R
    point's weight from the D array, 2ani_k.cuh:128) and for the 3-point
    kernels (which multiply every third point's weight into a running
    product)."""
    if not ref_cuda.available():
        pytest.skip("oracle/_ref/PCF_ref_cuda.out not built")
    box, dmax, P = 60.0, 20.0, 12
    three = kind.startswith("3")
    n = 1000 if three else 3000
    bins = 6 if kind == "3ani" else 10
    D, R = _lattice(n, 91, [1.0] if kind != "2iso" else [0.5, 1.0, 1.5, 2.0])
    run = ref_cuda.run_3pt_bpc if three else ref_cuda.run_2pt_bpc
    runs = {}
    for who, exe in (("ref", None), ("ours", OURS)):
        with tempfile.TemporaryDirectory() as wd:
            runs[who] = run(kind, D, R, box, bins, dmax, P, wd, exe=exe, timeout=300, bpc=False)
    for h in (("DDD", "RRR", "DDR", "DRR") if three else ("DD", "RR", "DR")):
        ref = runs["ref"][h]
        assert ref.sum() > 0, h
        got = runs["ours"][h].ravel()[:ref.size].reshape(ref.shape)
        assert np.array_equal(got, ref), h


def test_pcf_out_analytic_rr_equals_reference_program():
    """`2iso -bpc -a` (the periodic DD counted, RR and DR from the analytic
    formula, pcf2isoBPC.cuh:166-270) of the reference's program and of this
    PCF.out on a weighted lattice: the three files equal bit for bit.  (The
    3iso analytic path is not run: its DD2iso_forBPC bins a separation just
    below dmax with no bound check, 3isoBPC_k.cuh:1754-1757.)"""
    if not ref_cuda.available():
        pytest.skip("oracle/_ref/PCF_ref_cuda.out not built")
    D, _ = _lattice(3000, 93, [0.5, 1.0, 1.5, 2.0])
    res = {}
    for who, exe in (("ref", ref_cuda.EXE), ("ours", OURS)):
        with tempfile.TemporaryDirectory() as wd:
            for sub in ("data", "results", "run"):
                os.makedirs(os.path.join(wd, sub))
            ref_cuda._write(os.path.join(wd, "data", "data.dat"), D)
            ref_cuda._run_cli(exe, ["2iso", "-bpc", "-a", "-f", "data.dat", "-n", str(len(D)), "-b", "10",
                                    "-d", "20.0", "-s", "60.0", "-p", "12"], wd, 300)
            res[who] = {h: np.loadtxt(os.path.join(wd, "results", f"{h}iso_BPCanalytic_data.dat"))
                        for h in ("DD", "RR", "DR")}
    for h in ("DD", "RR", "DR"):
        assert res["ref"][h].sum() > 0, h
        assert np.array_equal(res["ours"][h], res["ref"][h]), (h, res["ours"][h], res["ref"][h])


@pytest.mark.parametrize("bpc", [False, True], ids=["plain", "periodic"])
def test_pcf_out_random_directory_equals_reference_program(bpc):
    """`2iso -rd DIR/` (one data catalog against every file of the directory,
    cuda/main.cu:157-192, pcf2iso.cuh:96-104 with its node and bin offsets per
    random file) of the reference's program and of this PCF.out (one batched
    launch) on weighted lattices: DD and every RR / DR file equal bit for bit.
    (2ani -rd is not run: the reference's XY2ani reads the R weight from the D
    array at an R index that passes D's end from the second random file on,
    2ani_k.cuh:128.)"""
    if not ref_cuda.available():
        pytest.skip("oracle/_ref/PCF_ref_cuda.out not built")
    n, w = 2000, [0.5, 1.0, 1.5, 2.0]
    D, R1 = _lattice(n, 95, w)
    _, R2 = _lattice(n, 96, w)
    _, R3 = _lattice(n, 97, w)
    res = {}
    for who, exe in (("ref", ref_cuda.EXE), ("ours", OURS)):
        with tempfile.TemporaryDirectory() as wd:
            for sub in ("data", "data/rands", "results", "run"):
                os.makedirs(os.path.join(wd, sub))
            ref_cuda._write(os.path.join(wd, "data", "data.dat"), D)
            for k, R in enumerate((R1, R2, R3)):
                ref_cuda._write(os.path.join(wd, "data", "rands", f"r{k}.dat"), R)
            ref_cuda._run_cli(exe, ["2iso"] + (["-bpc"] if bpc else []) + [
                "-f", "data.dat", "-rd", "rands/", "-n", str(n), "-b", "10", "-d", "20.0",
                "-s", "60.0", "-p", "12"], wd, 300)
            tag = "iso_BPC_" if bpc else "iso_"
            names = [f"DD{tag}data.dat"] + [f"{h}{tag}r{k}.dat" for k in range(3) for h in ("RR", "DR")]
            res[who] = {nm: np.loadtxt(os.path.join(wd, "results", nm)) for nm in names}
    for nm, ref in res["ref"].items():
        assert ref.sum() > 0, nm
        assert np.array_equal(res["ours"][nm], ref), nm
