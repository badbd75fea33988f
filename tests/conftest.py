import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "c_pp-library_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running CPU test")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Builds the checker library (and the product library when nvcc exists) once per session."""
    import oracle

    if not os.path.exists(oracle.PORT_LIB):
        oracle.build()
    elif not oracle.reference_available():
        tree = oracle.reference_tree()
        if tree and os.path.isdir(tree):
            oracle.build()
    yield


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def awcm_lib():
    import awcm

    if not os.path.exists(awcm.LIB_PATH):
        subprocess.run([sys.executable, os.path.join(PKG, "build.py")], check=True)
    return awcm
