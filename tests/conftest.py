import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "atom-mol-nonbo_b200")
for p in (PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

GOLDEN = os.path.join(ROOT, "tests", "golden", "hdplus_fixtures.npz")
FIXTURES = [f"inout_{w}_{k}" for w in (1, 2) for k in (500, 1000, 1500)]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    d = np.load(GOLDEN)

    def get(name):
        g = lambda k: d[f"{name}/{k}"]
        return dict(masses=g("masses"), charges=g("charges"), symmetry=str(g("symmetry")), K=int(g("K")),
                    energy=float(g("energy")), which=int(g("which")), tol=float(g("tol")),
                    invit=float(g("invit")), params=g("params"))

    return get
