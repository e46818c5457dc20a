import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 GPU (run with -m gpu)")
    config.addinivalue_line("markers", "slow: long-running")


def _have_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu():
    if not _have_gpu():
        pytest.skip("no GPU")
    from gpe_b200 import _lib
    _lib.load()
    return True


@pytest.fixture(scope="session", autouse=True)
def _oracle_threads():
    from oracle import pyoracle
    pyoracle.set_threads(int(os.environ.get("GPE_ORACLE_THREADS", str(os.cpu_count() or 1))))
