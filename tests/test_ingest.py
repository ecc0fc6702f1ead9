"""CPU: the parallel catalog reader (pcf_read_catalog) parses the reference's
text format exactly as ifstream >> float does, and the binary .f4 form
round-trips; the reader and PCF.out's histogram writers are pinned to the
reference's own open_files and save_histogram* (compiled in place)."""
import os

import numpy as np
import pytest

from desi_b200 import catalog


def _text(path, pts):
    with open(path, "w") as f:
        for p in pts:
            f.write(" ".join(repr(float(v)) for v in p) + "\n")


def test_text_reader_exact(tmp_path):
    rng = np.random.default_rng(1)
    pts = rng.uniform(0, 250, size=(20011, 4)).astype(np.float32)
    pts[::7, 3] = 1.0
    p = tmp_path / "c.dat"
    _text(p, pts)
    got, box = catalog.load(str(p), len(pts))
    assert np.array_equal(got, pts)
    assert box == np.ceil(pts[:, :3].max() + 1)
    few, _ = catalog.load(str(p), 100)
    assert np.array_equal(few, pts[:100])


def test_text_reader_ragged_whitespace(tmp_path):
    p = tmp_path / "r.dat"
    p.write_text("1 2 3 4\n\n  5\t6 7 8\r\n9 10 11 12")
    got, _ = catalog.load(str(p), 3)
    assert np.array_equal(got, np.arange(1, 13, dtype=np.float32).reshape(3, 4))


def test_short_or_missing_file(tmp_path):
    p = tmp_path / "s.dat"
    p.write_text("1 2 3 4\n")
    with pytest.raises(IOError):
        catalog.load(str(p), 2)
    with pytest.raises(IOError):
        catalog.load(str(tmp_path / "none.dat"), 1)


def test_f4_round_trip(tmp_path):
    pts = catalog.uniform(5000, 100.0, seed=3, weights="uniform")
    p = str(tmp_path / "c.f4")
    catalog.save_f4(p, pts)
    got, _ = catalog.load(p, 5000)
    assert np.array_equal(got, pts)


_REF_IO = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle", "_ref",
                       "libref_io.so")


@pytest.mark.skipif(not os.path.exists(_REF_IO), reason="needs oracle/_ref (reference tree at build)")
def test_text_reader_matches_reference_open_files(tmp_path):
    """The threaded reader against the reference's own open_files
    (cuda/create_grid.cuh:35-78, compiled in place): bit-equal points and the
    same automatic box, on decimals that do not round-trip to float32
    (17 significant digits), exponents, integers and mixed whitespace."""
    import oracle
    rng = np.random.default_rng(11)
    n = 30011
    v = rng.uniform(0.0, 250.0, size=(n, 4))
    v[:, 3] = rng.uniform(0.5, 1.5, n)
    rows = []
    for i, r in enumerate(v):
        if i % 5 == 0:
            s = " ".join(f"{x:.17g}" for x in r)
        elif i % 5 == 1:
            s = "\t".join(f"{x:.6e}" for x in r)
        elif i % 5 == 2:
            s = "  ".join(f"{x:.3f}" for x in r)
        elif i % 5 == 3:
            s = " ".join(str(int(x)) for x in r[:3]) + f" {r[3]:.9g}"
        else:
            s = " ".join(f"{x:.12g}" for x in r)
        rows.append(s)
    p = tmp_path / "mix.dat"
    p.write_text("\n".join(rows) + "\n")
    want, wbox = oracle.ref_read_catalog(str(p), n)
    got, box = catalog.load(str(p), n)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    assert box == wbox


@pytest.mark.skipif(not os.path.exists(_REF_IO), reason="needs oracle/_ref (reference tree at build)")
@pytest.mark.parametrize("dims", [1, 2, 3])
def test_histogram_files_match_reference_writers(tmp_path, dims):
    """PCF.out's histogram writers (desi_b200/csrc/pcf_io.hpp) write the same
    bytes as the reference's save_histogram1D/2D/3D (compiled in place) for
    counts, weighted sums, tiny values and zeros."""
    import subprocess

    import oracle
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    exe = str(tmp_path / "io_writer")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(root, "desi_b200", "csrc"),
                    "-I", os.path.join(root, "include"), os.path.join(root, "tests", "io_writer.cpp"),
                    "-o", exe], check=True)
    rng = np.random.default_rng(dims)
    bn = 7
    h = rng.uniform(0, 1e6, size=(bn,) * dims)
    flat = h.reshape(-1)
    flat[::5] = np.round(flat[::5] * 1e6)           # large integer counts
    flat[1::7] = rng.uniform(0, 1e-9, flat[1::7].size)  # tiny sums
    flat[2::9] = 0.0
    raw = tmp_path / "h.raw"
    raw.write_bytes(h.astype(np.float64).tobytes())
    (tmp_path / "results").mkdir()
    (tmp_path / "run").mkdir()
    subprocess.run([exe, str(dims), str(bn), str(raw), "ours.dat"], cwd=tmp_path / "run", check=True)
    want = tmp_path / "ref.dat"
    oracle.ref_save_histogram(h, str(want))
    assert (tmp_path / "results" / "ours.dat").read_bytes() == want.read_bytes()
