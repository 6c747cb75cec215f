import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle as O
    return O.lib()


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(autouse=True)
def _fresh_shape_cache(request):
    """GPU tests start without tuned launch shapes from earlier tests of the session."""
    if request.node.get_closest_marker("gpu") is not None:
        from spns_b200.hit import autotune_forget
        autotune_forget()
    yield
