import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "z80-optimizer_b200")
for p in (PKG, os.path.dirname(os.path.abspath(__file__))):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def ctx():
    import z80b
    c = z80b.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="session")
def O():
    import oracle_lib
    oracle_lib.build()
    return oracle_lib
