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


def test_program_runners_flags_and_files(tmp_path, monkeypatch):
    """run_2pt_bpc / run_3pt_bpc pass the reference's command line (with -bpc
    or not, -p, extra flags) and read back the files the reference names
    (<H><iso|ani>[_BPC]_<catalog>, create_grid.cuh:141-266)."""
    import subprocess
    seen = []

    class P:
        returncode = 0
        stdout = "Spent 12.5 miliseconds to compute and save all the histograms.\n"
        stderr = ""

    def fake_run(cmd, cwd, capture_output, text, timeout):
        seen.append(cmd)
        res = os.path.join(os.path.dirname(cwd), "results")
        kind, bpc = cmd[1], "-bpc" in cmd
        sfx = ("ani" if kind.endswith("ani") else "iso") + ("_BPC" if bpc else "")
        names = (("DDD", "RRR", "DDR", "DRR") if kind.startswith("3") else ("DD", "RR", "DR"))
        for h in names:
            cat = "data.dat" if h in ("DD", "DDD") else "rand.dat"
            np.savetxt(os.path.join(res, f"{h}{sfx}_{cat}"), np.full(8, len(h), float))
        return P()

    monkeypatch.setattr(subprocess, "run", fake_run)
    pts = np.ones((3, 4), np.float32)
    r = ref_cuda.run_3pt_bpc("3iso", pts, pts, 60.0, 2, 20.0, 6, str(tmp_path / "a"), extra=["-exact"])
    assert r["ms"] == 12.5 and r["DDD"].sum() == 24 and r["DRR"].size == 8
    assert seen[-1][1:3] == ["3iso", "-bpc"] and seen[-1][-3:] == ["-p", "6", "-exact"]
    r = ref_cuda.run_3pt_bpc("3ani", pts, pts, 60.0, 2, 20.0, 6, str(tmp_path / "b"), bpc=False)
    assert "-bpc" not in seen[-1] and r["RRR"].size == 8
    r = ref_cuda.run_2pt_bpc("2ani", pts, pts, 60.0, 2, 20.0, 6, str(tmp_path / "c"))
    assert seen[-1][1:3] == ["2ani", "-bpc"] and r["DR"].sum() == 16
    r = ref_cuda.run_2pt_bpc("2iso", pts, pts, 60.0, 2, 20.0, 6, str(tmp_path / "d"), bpc=False)
    assert "-bpc" not in seen[-1] and r["DD"].size == 8
