"""Shared test setup: the `gpu` marker, import paths for the package binding and the oracle."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "rak-lowmem-communities-cuda_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden", "golden.npz")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    return np.load(GOLDEN)


def golden_graph(z, name):
    import oracle as orc
    w = z[f"{name}/weights"] if f"{name}/weights" in z else None
    return orc.Graph(z[f"{name}/offsets"], z[f"{name}/targets"], w)
