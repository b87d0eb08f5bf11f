import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session", autouse=True)
def built_library():
    """libadabool.so up to date (compiles only what changed; needs nvcc)."""
    from adabool_b200 import build as B
    if B.LIB.exists():
        try:
            B.build()
        except Exception:
            pass  # a prebuilt library without a compiler (GPU box) is used as is
    else:
        B.build()
    return B.LIB


@pytest.fixture(scope="session")
def golden():
    return np.load(ROOT / "tests" / "golden" / "reference_vectors.npz")


def cuda_ok():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def dev():
    if not cuda_ok():
        pytest.skip("no CUDA device")
    import torch
    return torch.device("cuda", 0)
