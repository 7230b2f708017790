import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session", autouse=True)
def _oracle_built():
    """Builds the oracle libraries when their sources are newer (no-op on a prebuilt tree)."""
    from oracle import bindings
    if not os.path.exists(bindings.ORC_LIB) or (
            os.path.exists(os.path.join(ROOT, "oracle", "v3dba_oracle.c"))
            and os.path.getmtime(os.path.join(ROOT, "oracle", "v3dba_oracle.c")) > os.path.getmtime(bindings.ORC_LIB)):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "restate"], check=True,
                       stdout=subprocess.DEVNULL)
    yield
