import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: long-running")


def pytest_collection_modifyitems(config, items):
    try:
        import torch

        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(autouse=True)
def _rys_staging_waits(request):
    """After every GPU test: no bounded wait of the Rys kernels' table staging gave up."""
    yield
    if "gpu" not in request.keywords or "asuka_b200._lib" not in sys.modules:
        return
    lib = sys.modules["asuka_b200._lib"]
    if getattr(lib, "_LIB", None) is None:
        return
    rc = lib.lib().dfb_rys_error(1)
    assert rc <= 0, f"Rys table staging wait gave up (code {rc})"
