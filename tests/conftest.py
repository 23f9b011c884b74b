"""Shared pytest setup: the repository root on sys.path, the `gpu` marker,
and (re)building the CUDA library and the CPU oracle when their sources are
newer than the built files."""
import os
import shutil
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")
    config.addinivalue_line("markers", "slow: long-running case")


def _cuda_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


HAS_GPU = _cuda_available()


@pytest.fixture(scope="session", autouse=True)
def _built_libraries():
    import oracle
    from qd_imsrg_b200 import build as qbuild

    oracle.build()
    if shutil.which("nvcc") or os.path.exists("/usr/local/cuda/bin/nvcc"):
        qbuild.build()
    yield


@pytest.fixture
def gpu():
    if not HAS_GPU:
        pytest.skip("no CUDA device")
    return True
