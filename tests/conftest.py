import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")
    config.addinivalue_line("markers", "slow: long-running case")


_SNAPS = {}


def snapshot(name="small", **kw):
    """Cached synthetic snapshot (deterministic)."""
    from svdimager_b200 import synth
    key = (name, tuple(sorted(kw.items())))
    if key not in _SNAPS:
        _SNAPS[key] = synth.make_snapshot(name, **kw)
    return _SNAPS[key]


@pytest.fixture(scope="session")
def small_snapshot():
    return snapshot("small")


@pytest.fixture(scope="session")
def cuda_device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
