"""CPU: the parallel catalog reader (pcf_read_catalog) parses the reference's
text format exactly as ifstream >> float does, and the binary .f4 form
round-trips."""
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
