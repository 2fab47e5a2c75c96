import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA GPU")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def oracle_lib():
    from oracle import pyoracle
    return pyoracle


@pytest.fixture(scope="session")
def refhost():
    from oracle import pyoracle
    if not pyoracle.ReferenceHost.available():
        if not pyoracle.build_reference(gpu=False):
            pytest.skip("reference sources not available to build the host reference")
    return pyoracle.ReferenceHost()
