import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libwtbgpu.so")


def _have_gpu():
    try:
        import torch  # noqa: F401
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_ctx():
    from wantibexos_b200 import wtbgpu
    ctx = wtbgpu.Context(0)
    yield ctx
    ctx.close()
