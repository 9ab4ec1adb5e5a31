import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA kernels")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA GPU in this environment")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(autouse=True)
def _poison_shared_memory(request):
    """With LICA_POISON_SHARED=1, every GPU test starts from shared memory full of NaN, so a
    kernel that reads shared memory it has not written fails its parity check."""
    if os.environ.get("LICA_POISON_SHARED") == "1" and "gpu" in request.keywords:
        from lica_boiling1d_b200 import native
        native.poison_shared()
    yield
