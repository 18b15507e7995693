import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")
    config.addinivalue_line("markers", "reference: needs the reference sources and oracle/_ref")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    gpu = _has_gpu()
    from oracle import refdump
    ref = refdump.reference_available()
    for it in items:
        if "gpu" in it.keywords and not gpu:
            it.add_marker(pytest.mark.skip(reason="no CUDA GPU"))
        if "reference" in it.keywords and not ref:
            it.add_marker(pytest.mark.skip(reason="reference sources / oracle/_ref not available"))


@pytest.fixture(scope="session", autouse=True)
def _built():
    from master_thesis_b200 import build
    build.build()
    build.build_oracle()
