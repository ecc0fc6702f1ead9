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
Usage: python tests/golden/make_golden.py /path/to/reference
       python tests/golden/make_golden.py --fp64   (FP64-oracle histograms, see fp64_fixture)
The reference root comes from the argument or, failing that, the
PCF_REFERENCE_ROOT environment variable.
"""
import os
import sys

import numpy as np

REF = next((a for a in sys.argv[1:] if not a.startswith("--")), os.environ.get("PCF_REFERENCE_ROOT"))
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


if __name__ == "__main__" and "--fp64" not in sys.argv:
    if not REF:
        sys.exit("usage: make_golden.py /path/to/reference (or set PCF_REFERENCE_ROOT)")
    main()


def fp64_fixture():
    """FP64-oracle histograms of the golden configuration (plain 3iso,
    data.dat / rand0.dat, 32768 points, 30 bins, dmax 60, box 251 -- the
    reference's auto box ceil(max+1)) for the full-size GPU parity test."""
    sys.path.insert(0, os.path.dirname(os.path.dirname(OUT)))
    import oracle
    z = np.load(os.path.join(OUT, "catalogs.npz"))
    one = lambda a: np.ascontiguousarray(
        np.concatenate([a, np.ones((len(a), 1), np.float32)], 1).astype(np.float32))
    D, R = one(z["data"]), one(z["rand0"])
    kw = dict(box=251.0, bins=30, dmax=60.0)
    res = {
        "DDD": oracle.triplets_iso(D, **kw),
        "RRR": oracle.triplets_iso(R, **kw),
        "DDR": oracle.triplets_iso(D, R, **kw),
        "DRR": oracle.triplets_iso(R, D, **kw),
    }
    np.savez_compressed(os.path.join(OUT, "golden_3iso_fp64.npz"),
                        **{k: v.astype(np.int64) for k, v in res.items()})
    print({k: int(v.sum()) for k, v in res.items()})


if __name__ == "__main__" and "--fp64" in sys.argv:
    fp64_fixture()
