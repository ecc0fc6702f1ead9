"""Regenerate the committed fixtures of tests/golden from the reference tree.

Reads (needs the reference checkout; run in the development container):
  data/data.dat, data/rand0.dat          32768-point catalogs (unit weights)
  data/data_1K.dat, data/rand0_1K.dat    1000-point catalogs
  results/{DDD,DDR,DRR,RRR}iso.example   30^3 3iso histograms of the plain
                                         reference run on data.dat/rand0.dat
                                         (-n 32768 -b 30 -d 60)
Writes:
  catalogs.npz   float32 xyz of each catalog (weights are all 1 in the
                 reference files; checked here)
  golden_3iso.npz  int64 DDD, DDR, DRR, RRR (the .example values are integers)
Usage: python tests/golden/make_golden.py [/path/to/reference]
"""
import os
import sys

import numpy as np

REF = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
OUT = os.path.dirname(os.path.abspath(__file__))


def read(path):
    a = np.array(open(path, "rb").read().split(), dtype=np.float32).reshape(-1, 4)
    assert np.all(a[:, 3] == 1.0), path
    return a


def main():
    cats = {}
    for name in ("data", "rand0", "data_1K", "rand0_1K"):
        cats[name] = read(os.path.join(REF, "data", name + ".dat"))[:, :3].copy()
    np.savez_compressed(os.path.join(OUT, "catalogs.npz"), **cats)
    gold = {}
    for h in ("DDD", "DDR", "DRR", "RRR"):
        v = np.array(open(os.path.join(REF, "results", h + "iso.example")).read().split(),
                     dtype=np.float64)
        assert v.size == 30 ** 3 and np.all(v == np.round(v))
        gold[h] = v.astype(np.int64).reshape(30, 30, 30)
    np.savez_compressed(os.path.join(OUT, "golden_3iso.npz"), **gold)
    print({k: v.shape for k, v in cats.items()}, {k: int(v.sum()) for k, v in gold.items()})


if __name__ == "__main__":
    main()
