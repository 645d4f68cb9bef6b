import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "complab3d-gems_b200")
for p in (PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the product kernels")


@pytest.fixture(scope="session")
def clb():
    import clb as _clb
    _clb.lib()
    return _clb


@pytest.fixture(scope="session")
def oracle():
    import oracle as _o
    _o.lib()
    return _o
