"""Golden fixtures for the anisotropic 3-point oracle: the reference's own
3ani kernels run by oracle/_ref/ref_3ani.out (built from the reference tree,
its headers unmodified, by oracle/Makefile) on small seeded catalogs.
golden_3ani.npz holds the plain kernels (XXX3ani / XXY3ani,
cuda/kernels/3ani_k.cuh:8,109), golden_3ani_bpc.npz the periodic ones
(XXX3ani_BPC / XXY3ani_BPC, cuda/kernels/3aniBPC_k.cuh:210,959).  Needs a
GPU; run once:

    python tests/golden/make_golden_3ani.py [OUTDIR]   (default tests/golden)

The catalogs sit on integer lattices (data on even, randoms on odd
coordinates): every squared separation is then a small integer, exact in
the reference's FP32 sums and in the oracle's FP64 ones, and no data point
coincides with a random point (the reference bins a zero-length D-R side's
angle from 0/0).  Unit weights (the reference's kernels multiply the
weight of every third point into a running product).  dmax is a third of
the box: a pair is then in range through at most one periodic image, and a
triangle whose sides 12 and 31 are in range through their nearest images
has side 23 in range only through the image those two imply, which is the
case the periodic kernels' node projections enumerate."""
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
EXE = os.path.join(ROOT, "oracle", "_ref", "ref_3ani.out")
N, BOX, BINS, DMAX, PARTS = 1200, 60.0, 8, 20.0, 6


def catalogs():
    rng = np.random.default_rng(303)
    D = np.ones((N, 4), np.float32)
    R = np.ones((N, 4), np.float32)
    D[:, :3] = 2 * rng.integers(0, 30, size=(N, 3))      # 0, 2, ..., 58
    R[:, :3] = 2 * rng.integers(0, 30, size=(N, 3)) + 1  # 1, 3, ..., 59
    return D, R


def run(D, R, bpc):
    with tempfile.TemporaryDirectory() as d:
        fd, fr, fo = (os.path.join(d, x) for x in ("d.f4", "r.f4", "out.bin"))
        D.tofile(fd)
        R.tofile(fr)
        subprocess.run([EXE, fd, fr, str(N), str(BINS), repr(DMAX), str(PARTS), repr(BOX),
                        str(int(bpc)), fo], check=True, timeout=600)
        return np.fromfile(fo, dtype=np.float64).reshape(4, *(BINS,) * 5)


def main():
    D, R = catalogs()
    outdir = sys.argv[1] if len(sys.argv) > 1 else HERE
    for bpc, name in ((False, "golden_3ani.npz"), (True, "golden_3ani_bpc.npz")):
        h = run(D, R, bpc)
        np.savez_compressed(os.path.join(outdir, name), D=D, R=R, box=BOX, bins=BINS,
                            dmax=DMAX, partitions=PARTS, DDD=h[0], RRR=h[1], DDR=h[2], DRR=h[3])
        print(name, {k: float(v.sum()) for k, v in zip(("DDD", "RRR", "DDR", "DRR"), h)})


if __name__ == "__main__":
    sys.exit(main())
