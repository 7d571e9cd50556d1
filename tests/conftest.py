import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "chemrust-scf_b200")
ORACLE = os.path.join(ROOT, "oracle")
for p in (PKG, ORACLE, ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _ensure_built():
    import build  # chemrust-scf_b200/build.py
    import build_oracle
    build.build_library()
    build_oracle.build()


_ensure_built()


@pytest.fixture(scope="session")
def chfsi():
    import chfsi as m
    return m


@pytest.fixture(scope="session")
def oracle():
    import oracle as m
    return m


@pytest.fixture(scope="session")
def cfg0(chfsi):
    return chfsi.SyntheticSystem(config_index=0)
