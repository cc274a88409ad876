import os
import sys

import numpy as np
import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "ggms-distributed_b200")
for p in (REPO, PKG, os.path.join(REPO, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); runs the CUDA library")


@pytest.fixture(scope="session")
def ctx():
    import ggms_b200
    c = ggms_b200.Context(0)
    yield c
    c.close()


def to_device(a: np.ndarray):
    """numpy -> torch CUDA tensor holding the same bytes (uint32 travels as int32)."""
    import torch
    view = {np.dtype(np.uint32): np.int32}.get(a.dtype)
    t = torch.from_numpy(np.ascontiguousarray(a).view(view) if view else np.ascontiguousarray(a))
    return t.cuda()
