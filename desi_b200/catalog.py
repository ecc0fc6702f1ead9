"""Catalog I/O and seeded synthetic catalogs.

* :func:`read_catalog` / :func:`write_catalog`: the reference's text format,
  four whitespace-separated columns ``x y z w`` per row
  (cuda/create_grid.cuh:35-78, read with ``ifstream >>`` into floats);
  :func:`auto_box` reproduces its box rule ``ceil(max component + 1)``
  (create_grid.cuh:75).
* Synthetic generators stand in for survey catalogs (no dataset ships with
  the workload): uniform randoms and Neyman-Scott clustered data (uniform
  parents, Gaussian children, wrapped periodically), weights fixed at 1 or
  drawn from U(0.5, 1.5), all seeded.
"""
from __future__ import annotations

import math

import numpy as np


def read_catalog(path: str, n: int | None = None) -> np.ndarray:
    with open(path, "rb") as f:
        data = np.array(f.read().split(), dtype=np.float32)
    if data.size % 4:
        raise ValueError(f"{path}: expected 4 columns")
    pts = data.reshape(-1, 4)
    if n is not None:
        if len(pts) < n:
            raise ValueError(f"{path}: {len(pts)} rows < {n} requested")
        pts = pts[:n]
    return np.ascontiguousarray(pts)


def load(path: str, n: int) -> tuple[np.ndarray, float]:
    """First n points of a text or .f4 catalog through the library's parallel
    reader; returns (points, reference automatic box)."""
    import ctypes

    from . import _lib
    out = np.zeros((n, 4), np.float32)
    got = ctypes.c_int64()
    box = ctypes.c_float()
    rc = _lib.lib().pcf_read_catalog(path.encode(), n, out.ctypes.data_as(ctypes.c_void_p),
                                     ctypes.byref(got), ctypes.byref(box))
    if rc != 0:
        raise IOError(f"{path}: could not read {n} points (status {rc})")
    return out, box.value


def save_f4(path: str, pts: np.ndarray) -> None:
    np.ascontiguousarray(pts, dtype=np.float32).reshape(-1, 4).tofile(path)


def write_catalog(path: str, pts: np.ndarray) -> None:
    pts = np.asarray(pts, np.float32)
    with open(path, "w") as f:
        for p in pts:
            f.write(f"{p[0]!r} {p[1]!r} {p[2]!r} {p[3]!r}\n".replace("np.float32(", "").replace(")", ""))


def auto_box(*cats: np.ndarray) -> float:
    m = max(float(c[:, :3].max()) for c in cats)
    return float(math.ceil(m + 1))


def uniform(n: int, box: float, seed: int, weights: str = "unit") -> np.ndarray:
    rng = np.random.default_rng(seed)
    xyz = rng.uniform(0.0, box, size=(n, 3)).astype(np.float32)
    xyz = np.where(xyz >= np.float32(box), np.float32(0.0), xyz)
    return _with_weights(xyz, rng, weights)


def neyman_scott(n: int, box: float, seed: int, children: int = 64, sigma: float = 5.0,
                 weights: str = "unit") -> np.ndarray:
    """n points in ceil(n/children) Gaussian clusters around uniform parents,
    wrapped into [0, box)."""
    rng = np.random.default_rng(seed)
    parents = rng.uniform(0.0, box, size=(int(math.ceil(n / children)), 3))
    idx = np.repeat(np.arange(len(parents)), children)[:n]
    xyz = parents[idx] + rng.normal(0.0, sigma, size=(n, 3))
    xyz = np.mod(xyz, box).astype(np.float32)
    xyz = np.where(xyz >= np.float32(box), np.float32(0.0), xyz)
    return _with_weights(xyz, rng, weights)


def _with_weights(xyz, rng, weights):
    n = len(xyz)
    if weights == "unit":
        w = np.ones((n, 1), np.float32)
    elif weights == "uniform":
        w = rng.uniform(0.5, 1.5, size=(n, 1)).astype(np.float32)
    else:
        raise ValueError(weights)
    return np.ascontiguousarray(np.concatenate([xyz, w], axis=1).astype(np.float32))
