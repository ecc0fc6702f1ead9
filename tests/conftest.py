import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and libpcf.so")
    config.addinivalue_line("markers", "slow: long-running CPU check")


def _cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def with_unit_w(xyz):
    return np.ascontiguousarray(
        np.concatenate([xyz, np.ones((len(xyz), 1), np.float32)], axis=1).astype(np.float32))


@pytest.fixture(scope="session")
def catalogs():
    z = np.load(os.path.join(GOLDEN, "catalogs.npz"))
    return {k: with_unit_w(z[k]) for k in z.files}


@pytest.fixture(scope="session")
def golden_3iso():
    z = np.load(os.path.join(GOLDEN, "golden_3iso.npz"))
    return {k: z[k].astype(np.float64) for k in z.files}


@pytest.fixture(scope="session")
def ctx():
    from desi_b200 import api
    c = api.Context(0)
    yield c
    c.close()
