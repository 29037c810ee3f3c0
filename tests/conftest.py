import os
import sys

import numpy as np
import pytest

ROOT = os.path.abspath(os.path.join(os.path.dirname(__file__), ".."))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden", "redrock_golden.npz")


def redrock_dir():
    """Directory holding an unmodified redrock package, or None: the
    reference install at baseline/_ref (pip --target), else $REDROCK_PY."""
    for d in (os.path.join(ROOT, "baseline", "_ref"), os.environ.get("REDROCK_PY")):
        if d and os.path.exists(os.path.join(d, "redrock", "zscan.py")):
            return d
    return None


def redrock_test_data(name):
    """Path of a file in redrock's own test data, or None when absent."""
    d = redrock_dir()
    p = None if d is None else os.path.join(d, "redrock", "test", "data", name)
    return p if p and os.path.exists(p) else None


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def golden():
    return dict(np.load(GOLDEN))


def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
