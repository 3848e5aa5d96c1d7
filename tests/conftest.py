import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parent.parent
GOLDEN = REPO / "tests" / "golden"
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libtpo")


def pytest_collection_modifyitems(config, items):
    try:
        import torch
        have_cuda = torch.cuda.is_available()
    except Exception:  # pragma: no cover
        have_cuda = False
    if have_cuda:
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


def golden(name: str):
    return np.load(GOLDEN / f"{name}.npz")


@pytest.fixture(scope="session")
def tpo_built():
    """Build libtpo if stale (the GPU machines carry the prebuilt .so)."""
    from toptimization_b200.csrc import build
    build.build()
    from toptimization_b200 import _lib
    return _lib.load()
