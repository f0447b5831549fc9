import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "tt-toolbox_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libttgpu.so")


@pytest.fixture(scope="session")
def ctx():
    import ttgpu
    c = ttgpu.Context(int(os.environ.get("TTG_DEVICE", "0")))
    yield c
    c.close()
