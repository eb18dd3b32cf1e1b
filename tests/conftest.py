import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
TESTS = os.path.dirname(os.path.abspath(__file__))
if TESTS not in sys.path:
    sys.path.insert(0, TESTS)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session")
def product_lib():
    """The CUDA library (built in-tree if it is missing)."""
    import psp_b200
    if not os.path.exists(psp_b200.LIB_PATH):
        from psp_b200 import build
        build.build()
    return psp_b200.lib()


def oracle_for(disc, damping=7.0, planes=4, cutoff=12):
    import oracle
    od = oracle.make_disc(disc.omega, disc.nx, disc.ny, disc.nz, disc.wx, disc.wy, disc.wz,
                          bcs=(disc.frontBC, disc.rightBC, disc.backBC, disc.leftBC, disc.topBC),
                          pml=(disc.bx, disc.by, disc.bz), sigma=disc.sigmax)
    return oracle.Oracle(od, damping, planes, cutoff)


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))
