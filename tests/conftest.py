import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _ensure_built():
    """Build the oracle and the product library when they are missing (CPU
    cross-compilation works without a GPU)."""
    if not os.path.exists(os.path.join(ROOT, "oracle", "liboracle_bcr.so")):
        subprocess.run(["make", "-s", "liboracle_bcr.so"], cwd=os.path.join(ROOT, "oracle"), check=True)
    if not os.path.exists(os.path.join(ROOT, "alglin_b200", "libalglin_b200.so")):
        subprocess.run(["make", "-s"], cwd=os.path.join(ROOT, "alglin_b200"), check=True)


_ensure_built()


@pytest.fixture(scope="session")
def has_gpu():
    import torch
    return torch.cuda.is_available()
