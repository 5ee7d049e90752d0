import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

REFERENCE = os.environ.get("MDFF_REFERENCE", "/root/reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the engine kernels")


def has_reference():
    return os.path.isdir(os.path.join(REFERENCE, "examples"))


@pytest.fixture(scope="session", autouse=True)
def _built():
    import oracle
    if not os.path.exists(os.path.join(ROOT, "oracle", "_build", "liboracle.so")):
        oracle.build()
    import mdff_b200
    if not os.path.exists(mdff_b200.LIB_PATH):
        mdff_b200.build()
    yield


def gpu_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)
