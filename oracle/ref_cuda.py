"""Runner of the reference's own CUDA program (baseline infrastructure only).

`oracle/Makefile` target `ref_cuda` builds cuda/main.cu of the reference
tree, unmodified, with nvcc for sm_100a into oracle/_ref/PCF_ref_cuda.out.
This module runs it on given catalogs the way its CLI expects them:

* catalogs are read as text rows "x y z w" from ../data/<name> relative to
  the working directory (cuda/create_grid.cuh:35-78, open_files);
* histograms are written as text to ../results/<kind>_<name>
  (create_grid.cuh:141-160, save_histogram1D);
* the time it prints ("Spent <ms> miliseconds ...", pcf2isoBPC.cuh:137-139)
  is a CUDA-event interval around the kernels, the D2H copies and the file
  writes.

Driven: the periodic paths `2iso -bpc`, `3iso -bpc` and `3ani -bpc`, one
random file.  Their kernels guard every histogram index (the `bin>(bn-1)`
checks before each atomicAdd in 2isoBPC_k.cuh, 3isoBPC_k.cuh and
3aniBPC_k.cuh) and read points only inside node ranges.  The host grid
(make_nodos, create_grid.cuh:130-133) indexes cells by (int)(x / size_node)
without a clamp, so coordinates are kept at least 1e-3 inside the box.  The
`-a` path and the anisotropic pair cross kernels are not run.
"""
import os
import re
import subprocess
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
EXE = os.path.join(HERE, "_ref", "PCF_ref_cuda.out")


def available():
    return os.path.exists(EXE)


def inside_box(pts, box, margin=1e-3):
    """The catalog with coordinates clamped to [0, box - margin]."""
    out = np.array(pts, dtype=np.float32, copy=True)
    out[:, :3] = np.clip(out[:, :3], 0.0, np.float32(box - margin))
    return out


def _write(path, pts):
    with open(path, "w") as f:
        for x, y, z, w in pts.astype(np.float64):
            f.write(f"{x:.9g} {y:.9g} {z:.9g} {w:.9g}\n")


def run_2iso_bpc(D, R, box, bins, dmax, workdir, timeout=600):
    """Runs `2iso -bpc` on D (data) and R (one random catalog), both with
    len(D) == len(R) rows; returns {"ms", "wall_s", "DD", "RR", "DR", "stdout"}
    (wall_s: the whole process, reading, host grid and device set-up included)."""
    if len(D) != len(R):
        raise ValueError("the reference reads -n rows from each file")
    for sub in ("data", "results", "run"):
        os.makedirs(os.path.join(workdir, sub), exist_ok=True)
    _write(os.path.join(workdir, "data", "data.dat"), D)
    _write(os.path.join(workdir, "data", "rand.dat"), R)
    cmd = [EXE, "2iso", "-bpc", "-f", "data.dat", "-r", "rand.dat", "-n", str(len(D)),
           "-b", str(int(bins)), "-d", repr(float(dmax)), "-s", repr(float(box))]
    t0 = time.perf_counter()
    p = subprocess.run(cmd, cwd=os.path.join(workdir, "run"), capture_output=True, text=True,
                       timeout=timeout)
    wall = time.perf_counter() - t0
    if p.returncode != 0:
        raise RuntimeError(f"reference CUDA program exited {p.returncode}: {p.stdout[-300:]} {p.stderr[-300:]}")
    m = re.search(r"Spent\s+([0-9.eE+-]+)\s+miliseconds", p.stdout)
    if not m:
        raise RuntimeError("no timer line in the reference's output: " + p.stdout[-300:])
    res = {"ms": float(m.group(1)), "wall_s": wall, "stdout": p.stdout}
    for kind in ("DD", "RR", "DR"):
        name = {"DD": "data.dat", "RR": "rand.dat", "DR": "rand.dat"}[kind]
        res[kind] = np.loadtxt(os.path.join(workdir, "results", f"{kind}iso_BPC_{name}"))
    return res


def _run_cli(exe, args, workdir, timeout):
    t0 = time.perf_counter()
    p = subprocess.run([exe] + args, cwd=os.path.join(workdir, "run"), capture_output=True,
                       text=True, timeout=timeout)
    wall = time.perf_counter() - t0
    if p.returncode != 0:
        raise RuntimeError(f"{os.path.basename(exe)} exited {p.returncode}: {p.stdout[-300:]} {p.stderr[-300:]}")
    m = re.search(r"Spent\s+([0-9.eE+-]+)\s+miliseconds", p.stdout)
    return (float(m.group(1)) if m else None), wall


def run_3pt_bpc(kind, D, R, box, bins, dmax, partitions, workdir, exe=None, timeout=600, extra=(),
                bpc=True):
    """Runs `<kind> -bpc -p partitions` (kind "3iso" or "3ani") of the
    reference's CUDA program, or of another program with the same command
    line (exe, e.g. this library's PCF.out), on D and one random catalog R
    (len(D) == len(R)); returns {"ms", "wall_s", "DDD", "RRR", "DDR", "DRR"}
    with each histogram as written: bins^3 values (the reference's 3ani
    writer keeps the first bins^3 of its bins^5 histogram, pcf3aniBPC.cuh:123,
    create_grid.cuh:197) or, for a writer of the full 3ani histogram, all
    bins^5.  The reference's kernels read points only inside node ranges and
    check every bin index (3isoBPC_k.cuh:80-85, 3aniBPC_k.cuh:77-85); its
    host grid does not clamp cell indices, so coordinates are kept 1e-3 inside
    the box by the caller (inside_box).  extra: more command-line flags (this
    library's -exact); bpc=False runs the plain path (`<kind>` without -bpc:
    XXX3iso / XXY3iso, XXX3ani / XXY3ani)."""
    if len(D) != len(R):
        raise ValueError("the reference reads -n rows from each file")
    exe = exe or EXE
    for sub in ("data", "results", "run"):
        os.makedirs(os.path.join(workdir, sub), exist_ok=True)
    _write(os.path.join(workdir, "data", "data.dat"), D)
    _write(os.path.join(workdir, "data", "rand.dat"), R)
    args = [kind] + (["-bpc"] if bpc else []) + [
        "-f", "data.dat", "-r", "rand.dat", "-n", str(len(D)), "-b", str(int(bins)),
        "-d", repr(float(dmax)), "-s", repr(float(box)), "-p", str(int(partitions))] + list(extra)
    ms, wall = _run_cli(exe, args, workdir, timeout)
    res = {"ms": ms, "wall_s": wall}
    sfx = ("ani" if kind == "3ani" else "iso") + ("_BPC" if bpc else "")
    for h in ("DDD", "RRR", "DDR", "DRR"):
        name = "data.dat" if h == "DDD" else "rand.dat"
        res[h] = np.loadtxt(os.path.join(workdir, "results", f"{h}{sfx}_{name}")).ravel()
    return res


def run_2pt_bpc(kind, D, R, box, bins, dmax, partitions, workdir, exe=None, timeout=600, bpc=True):
    """Runs `<kind> -bpc -p partitions` (kind "2iso" or "2ani") of the
    reference's CUDA program, or of another program with the same command
    line (exe), on D and one random catalog R; returns {"ms", "wall_s", "DD",
    "RR", "DR"} as written (bins values, or bins x bins for 2ani).  The
    reference's XY2ani_BPC weights most pairs by an unset variable
    (2aniBPC_k.cuh:372,410,429), so its 2ani DR is not a result.  bpc=False
    runs the plain path (XX2iso / XY2iso, XX2ani / XY2ani), whose XY2ani
    takes the weight of its R point from the D array at the R index
    (2ani_k.cuh:128): in bounds with one random file of the same length, so
    its DR is a result with unit weights only."""
    if len(D) != len(R):
        raise ValueError("the reference reads -n rows from each file")
    exe = exe or EXE
    for sub in ("data", "results", "run"):
        os.makedirs(os.path.join(workdir, sub), exist_ok=True)
    _write(os.path.join(workdir, "data", "data.dat"), D)
    _write(os.path.join(workdir, "data", "rand.dat"), R)
    args = [kind] + (["-bpc"] if bpc else []) + [
        "-f", "data.dat", "-r", "rand.dat", "-n", str(len(D)), "-b", str(int(bins)),
        "-d", repr(float(dmax)), "-s", repr(float(box)), "-p", str(int(partitions))]
    ms, wall = _run_cli(exe, args, workdir, timeout)
    res = {"ms": ms, "wall_s": wall}
    sfx = ("ani" if kind == "2ani" else "iso") + ("_BPC" if bpc else "")
    for h in ("DD", "RR", "DR"):
        name = "data.dat" if h == "DD" else "rand.dat"
        res[h] = np.loadtxt(os.path.join(workdir, "results", f"{h}{sfx}_{name}"))
    return res
