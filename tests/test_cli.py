"""The PCF.out drop-in CLI and the reference-signature C++ entry points.

CPU: argument handling (messages and exit codes of cuda/main.cu:99-117).
GPU: PCF.out runs in the reference's directory layout (cwd cuda/, inputs in
../data/, outputs in ../results/) and writes the reference's file names and
text formats; values match the FP64 oracle.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle
from desi_b200 import catalog

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "desi_b200", "PCF.out")


def _run(args, cwd, check=True):
    p = subprocess.run([CLI] + args, cwd=cwd, capture_output=True, text=True, timeout=300)
    if check and p.returncode != 0:
        raise AssertionError(p.stdout + p.stderr)
    return p


@pytest.fixture
def layout(tmp_path):
    for d in ("data", "results", "cuda", "data/rands"):
        (tmp_path / d).mkdir(parents=True, exist_ok=True)
    return tmp_path


def _write(path, pts):
    np.savetxt(path, pts, fmt="%.9g")


def _read(path, n=None):
    return np.array(open(path).read().split(), dtype=np.float64)


def test_help_and_argument_errors(layout):
    assert "Use: ./PCF" in _run(["--help"], layout / "cuda").stdout
    p = _run(["2iso", "-f", "x"], layout / "cuda", check=False)
    assert p.returncode == 1 and "Invalid <calc_type>" in p.stdout
    p = _run(["2iso", "-f", "d.dat", "-r", "r.dat", "-b", "10", "-d", "5"], layout / "cuda", check=False)
    assert p.returncode == 1 and "Missing number of points" in p.stdout
    p = _run(["2iso", "-f", "d.dat", "-n", "10", "-b", "10", "-d", "5"], layout / "cuda", check=False)
    assert p.returncode == 1 and "Missing random file" in p.stdout
    p = _run(["2iso", "-f", "nothere.dat", "-r", "r.dat", "-n", "10", "-b", "10", "-d", "5"],
             layout / "cuda", check=False)
    assert p.returncode == 1 and "Failed to load the file" in p.stdout


def _cats(layout, n=1500, box=100.0):
    D = catalog.neyman_scott(n, box - 2, seed=61)
    R = catalog.uniform(n, box - 2, seed=62)
    R2 = catalog.uniform(n, box - 2, seed=63)
    D = np.round(D.astype(np.float64), 5).astype(np.float32)  # exact text round trip
    R = np.round(R.astype(np.float64), 5).astype(np.float32)
    R2 = np.round(R2.astype(np.float64), 5).astype(np.float32)
    _write(layout / "data" / "d.dat", D)
    _write(layout / "data" / "r.dat", R)
    _write(layout / "data" / "rands" / "ra.dat", R)
    _write(layout / "data" / "rands" / "rb.dat", R2)
    back = lambda p: np.loadtxt(p, dtype=np.float32)
    return back(layout / "data" / "d.dat"), back(layout / "data" / "r.dat"), back(layout / "data" / "rands" / "rb.dat")


@pytest.mark.gpu
def test_cli_2iso_2ani_plain_bpc_rd(layout):
    D, R, R2 = _cats(layout)
    box = 100.0
    n = len(D)
    _run(["2iso", "-n", str(n), "-f", "d.dat", "-r", "r.dat", "-b", "20", "-d", "30", "-s", str(box)],
         layout / "cuda")
    res = layout / "results"
    assert np.array_equal(_read(res / "DDiso_d.dat"), oracle.pairs(D, box=box, bins=20, dmax=30.0))
    assert np.array_equal(_read(res / "DRiso_r.dat"), oracle.pairs(D, R, box=box, bins=20, dmax=30.0))
    _run(["2ani", "-n", str(n), "-f", "d.dat", "-rd", "rands/", "-b", "12", "-d", "30", "-bpc",
          "-s", str(box)], layout / "cuda")
    # -rd: both random files through one batched launch
    kw = dict(box=box, bins=12, dmax=30.0, ani=True, bpc=True)
    got = _read(res / "RRani_BPC_rb.dat").reshape(12, 12)
    assert np.array_equal(got, oracle.pairs(R2, **kw))
    assert np.array_equal(_read(res / "DRani_BPC_ra.dat").reshape(12, 12), oracle.pairs(D, R, **kw))
    assert np.array_equal(_read(res / "DRani_BPC_rb.dat").reshape(12, 12), oracle.pairs(D, R2, **kw))
    assert np.array_equal(_read(res / "RRani_BPC_ra.dat").reshape(12, 12), oracle.pairs(R, **kw))
    _run(["2iso", "-n", str(n), "-f", "d.dat", "-rd", "rands/", "-b", "20", "-d", "30", "-s", str(box)],
         layout / "cuda")
    for lab, RR in (("ra", R), ("rb", R2)):
        assert np.array_equal(_read(res / f"RRiso_{lab}.dat"), oracle.pairs(RR, box=box, bins=20, dmax=30.0))
        assert np.array_equal(_read(res / f"DRiso_{lab}.dat"),
                              oracle.pairs(D, RR, box=box, bins=20, dmax=30.0))
    # text layout of the 2-D writer: bins lines of bins values each
    lines = open(res / "DDani_BPC_d.dat").read().split("\n")
    assert len(lines[0].split()) == 12
    _run(["2iso", "-n", str(n), "-f", "d.dat", "-b", "20", "-d", "30", "-bpc", "-a", "-s", str(box)],
         layout / "cuda")
    rr = _read(res / "RRiso_BPCanalytic_d.dat")
    # the writers keep 12 significant digits (setprecision(12))
    np.testing.assert_allclose(rr, oracle.analytic_rr(20, n, box, 30.0), rtol=1e-11)
    dd = _read(res / "DDiso_BPCanalytic_d.dat")
    assert np.array_equal(dd, oracle.pairs(D, box=box, bins=20, dmax=30.0, bpc=True, ds_exact=True))


@pytest.mark.gpu
def test_cli_3iso_and_file_format(layout):
    D, R, _ = _cats(layout, n=800)
    box = 100.0
    _run(["3iso", "-n", "800", "-f", "d.dat", "-r", "r.dat", "-b", "8", "-d", "20", "-s", str(box)],
         layout / "cuda")
    res = layout / "results"
    text = open(res / "DDDiso_d.dat").read()
    # save_histogram3D: 8 rows of 8 values then "\n\n" per slab
    assert text.count("\n") == 8 * 8 + 8 * 2
    got = _read(res / "DDRiso_r.dat").reshape(8, 8, 8)
    assert np.array_equal(got, oracle.triplets_iso(D, R, box=box, bins=8, dmax=20.0))


@pytest.mark.gpu
@pytest.mark.parametrize("exact", [True, False], ids=["exact", "reference_gates"])
def test_cli_3iso_rd_batched(layout, exact):
    """PCF.out 3iso -rd -bpc: DDD and every random file's RRR / DDR / DRR.
    With -exact from one batched launch, each equal to the oracle's count of
    every triangle in range; by default per call through the reference's node
    gates on its -p grid (35 nodes per side), equal to the oracle's
    restatement of those gates (PCF_REF_NODE_GATES)."""
    D, R, R2 = _cats(layout, n=700)
    box = 100.0
    _run(["3iso", "-n", "700", "-f", "d.dat", "-rd", "rands/", "-b", "8", "-d", "20", "-bpc",
          "-s", str(box)] + (["-exact"] if exact else []), layout / "cuda")
    res = layout / "results"
    kw = dict(box=box, bins=8, dmax=20.0, bpc=True, ref_gates=0 if exact else 35)
    rd = lambda name: _read(res / name).reshape(8, 8, 8)  # noqa: E731
    assert np.array_equal(rd("DDDiso_BPC_d.dat"), oracle.triplets_iso(D, **kw))
    for lab, RR in (("ra", R), ("rb", R2)):
        assert np.array_equal(rd(f"RRRiso_BPC_{lab}.dat"), oracle.triplets_iso(RR, **kw))
        assert np.array_equal(rd(f"DDRiso_BPC_{lab}.dat"), oracle.triplets_iso(D, RR, **kw))
        assert np.array_equal(rd(f"DRRiso_BPC_{lab}.dat"), oracle.triplets_iso(RR, D, **kw))


@pytest.mark.gpu
def test_cli_3ani_writes_every_bin(layout):
    """PCF.out 3ani writes the full bins^5 histogram (the reference's writer
    stops at bins^3 values, cuda/pcf3ani.cuh:123): bins^4 lines of bins
    values, in [b12][b31][b23][t12][t31] order, equal to the oracle."""
    D, R, _ = _cats(layout, n=300)
    box, bins = 100.0, 4
    _run(["3ani", "-n", "300", "-f", "d.dat", "-r", "r.dat", "-b", str(bins), "-d", "25",
          "-s", str(box)], layout / "cuda")
    res = layout / "results"
    text = open(res / "DDDani_d.dat").read()
    rows = [ln for ln in text.split("\n") if ln.strip()]
    assert len(rows) == bins ** 4 and all(len(r.split()) == bins for r in rows)
    got = np.array(text.split(), dtype=np.float64).reshape((bins,) * 5)
    want = oracle.triplets_ani(D, box=box, bins=bins, dmax=25.0)
    assert want.sum() > 0
    assert np.array_equal(got, want)
    got = _read(res / "DDRani_r.dat").reshape((bins,) * 5)
    assert np.array_equal(got, oracle.triplets_ani(D, R, box=box, bins=bins, dmax=25.0))


@pytest.mark.gpu
def test_legacy_signatures(layout, tmp_path):
    exe = str(tmp_path / "legacy_driver")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    "-I", "/usr/local/cuda/include", os.path.join(ROOT, "tests", "legacy_driver.cpp"),
                    "-o", exe, "-L", os.path.join(ROOT, "desi_b200"), "-lpcf",
                    "-L", "/usr/local/cuda/lib64", "-lcudart",
                    "-Wl,-rpath," + os.path.join(ROOT, "desi_b200")], check=True)
    D, R, _ = _cats(layout, n=900)
    d, r = str(layout / "data" / "d.dat"), str(layout / "data" / "r.dat")
    for kind in ("2iso", "2aniBPC", "3iso", "2isoBPCa", "3isoBPC"):
        subprocess.run([exe, kind, d, r, "900", "10", "20", "100"], cwd=layout / "cuda", check=True,
                       timeout=300)
    res = layout / "results"
    # pcf_3isoBPC counts through the reference's node gates on the caller's
    # grid (size_node = box / 10 in the driver)
    assert np.array_equal(_read(res / "RRRiso_BPC_rand").reshape(10, 10, 10),
                          oracle.triplets_iso(R, box=100.0, bins=10, dmax=20.0, bpc=True, ref_gates=10))
    assert np.array_equal(_read(res / "DDiso_data"), oracle.pairs(D, box=100.0, bins=10, dmax=20.0))
    assert np.array_equal(_read(res / "DRani_BPC_rand").reshape(10, 10),
                          oracle.pairs(D, R, box=100.0, bins=10, dmax=20.0, ani=True, bpc=True))
    assert np.array_equal(_read(res / "RRRiso_rand").reshape(10, 10, 10),
                          oracle.triplets_iso(R, box=100.0, bins=10, dmax=20.0))
    assert (res / "RRiso_BPCanalytic_data").exists()
