import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (os.path.join(ROOT, "rgbd-flow_b200"), os.path.join(ROOT, "tests"), ROOT):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle_binding as ob
    ob.build_oracle()
    return ob.oracle()


@pytest.fixture(scope="session")
def ctx():
    import rgbdflow as rf
    c = rf.Context(0)
    yield c
    c.close()
