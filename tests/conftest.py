import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "smoq.jl_b200"), os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a); runs the CUDA library")


@pytest.fixture(scope="session")
def built():
    import build  # smoq.jl_b200/build.py
    build.build_cuda()
    build.build_oracle()
    return True


@pytest.fixture(scope="session")
def ctx(built):
    import pysmoq
    c = pysmoq.Context(0)
    yield c
    c.close()
