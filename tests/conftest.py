"""Shared pytest configuration: the `gpu` marker and import paths."""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); parity tests through the C ABI")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # pragma: no cover - torch missing
        return False


@pytest.fixture(scope="session")
def require_gpu():
    if not cuda_available():
        pytest.fail("this test needs a CUDA device; run it with -m gpu on a GPU host")
