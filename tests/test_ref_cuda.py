"""Host side of the reference-CUDA runner (oracle/ref_cuda.py): the catalog
files it writes round-trip to the same float32 values, the box clamp keeps
every coordinate inside the reference's unclamped cell grid, and its timer
line is parsed.  The program itself runs only on a GPU, opt-in from bench.py."""
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from oracle import ref_cuda  # noqa: E402


def test_catalog_files_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    pts = rng.uniform(0, 250, (1000, 4)).astype(np.float32)
    pts[:, 3] = rng.uniform(0.5, 1.5, 1000).astype(np.float32)
    path = tmp_path / "c.dat"
    ref_cuda._write(str(path), pts)
    back = np.loadtxt(str(path)).astype(np.float32)
    assert np.array_equal(back, pts)


def test_inside_box_clamp():
    box = 250.0
    pts = np.array([[249.99999, 0.0, 125.0, 1.0], [-0.0, 250.0, 3.0, 2.0]], np.float32)
    out = ref_cuda.inside_box(pts, box)
    assert np.all(out[:, :3] <= np.float32(box - 1e-3)) and np.all(out[:, :3] >= 0)
    assert np.array_equal(out[:, 3], pts[:, 3])
    # every clamped coordinate bins below the reference's 35 partitions
    size_node = np.float32(box) / np.float32(35)
    assert np.all((out[:, :3] / size_node).astype(np.int64) < 35)


def test_timer_line_parsed(tmp_path, monkeypatch):
    import subprocess

    class P:
        returncode = 0
        stdout = "Succesfully readed the data.\nSpent 237.5 miliseconds to compute and save all the histograms.\n"
        stderr = ""

    def fake_run(cmd, cwd, capture_output, text, timeout):
        res = os.path.join(os.path.dirname(cwd), "results")
        for kind, name in (("DD", "data.dat"), ("RR", "rand.dat"), ("DR", "rand.dat")):
            np.savetxt(os.path.join(res, f"{kind}iso_BPC_{name}"), np.arange(4.0))
        return P()

    monkeypatch.setattr(subprocess, "run", fake_run)
    pts = np.zeros((4, 4), np.float32)
    r = ref_cuda.run_2iso_bpc(pts, pts, 250.0, 4, 80.0, str(tmp_path))
    assert r["ms"] == 237.5 and r["DD"].shape == (4,)
