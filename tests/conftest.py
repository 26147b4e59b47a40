import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the library's kernels")


@pytest.fixture(scope="session")
def gpu_ctx():
    import dplasma_b200 as db
    ctx = db.Context(0)
    yield ctx
    ctx.close()
